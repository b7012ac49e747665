"""Extract the known-answer vectors that pin the linear-solve hot path from the
kelofm/cie test sources and write them as small JSON fixtures beside this script.

Run in a container that has the reference checkout (default location below, or
pass it as the first argument).  The fixtures are committed; nothing at test time
reads the reference.

Sources (paths relative to the reference project root):
  * libraries/linalg/packages/solvers/test/SYCLSpace_test.cpp:28-47   innerProduct sizes
  * libraries/linalg/packages/solvers/test/SYCLSpace_test.cpp:70-138  add / scale cases
  * libraries/linalg/packages/solvers/test/SYCLSpace_test.cpp:141-186 SpMV known answer
  * libraries/linalg/packages/solvers/test/SYCLSpace_test.cpp:188-246 masked SpMV known answer
  * libraries/fem/packages/integrands/test/LinearIsotropicStiffnessIntegrand_test.cpp:20-93
  * libraries/fem/packages/numeric/test/GaussLegendreQuadrature_test.cpp:14-152
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def numbers(text):
    return [float(x) for x in re.findall(r"[-+]?\d+(?:\.\d+)?(?:[eE][-+]?\d+)?", text)]


def vector_literal(block, name):
    m = re.search(r"std::vector<[^>]+>\s+" + name + r"\s*\{([^}]*)\}", block)
    return numbers(m.group(1))


def space_cases():
    src = read("libraries/linalg/packages/solvers/test/SYCLSpace_test.cpp")
    out = {}
    # innerProduct: sizes 1e1+1 ... 1e7+7, iota . (-1) = -n(n-1)/2
    m = re.search(r"for \(const std::size_t size : \{([^}]*)\}\)", src)
    sizes = [int(round(eval(s))) for s in m.group(1).split(",")]
    out["inner_product"] = [{"size": n, "expected": -n * (n - 1) / 2.0} for n in sizes]
    # add / scale use sizes {1e1 ... 1e5} and closed-form expectations
    m = re.search(r'CASE_INIT\("add"\)\s*for \(std::size_t size : \{([^}]*)\}\)', src)
    out["elementwise_sizes"] = [int(round(eval(s))) for s in m.group(1).split(",")]
    out["add"] = {"target_factor": 1e1, "first_scale": 1e2, "second_scale": 1.0}
    out["scale_uniform"] = {"factor": 2.0}
    out["scale_componentwise"] = {"target_factor": 1e1, "scale": 1e2}

    def spmv_block(tag):
        start = src.index('CASE_INIT("%s")' % tag)
        end = src.index("} // SpMV", start)
        return src[start:end]

    for key, tag in (("spmv", "SpMV"), ("masked_spmv", "SpMV (masked)")):
        b = spmv_block(tag)
        case = {
            "entries": vector_literal(b, "entries"),
            "column_indices": [int(x) for x in vector_literal(b, "columnIndices")],
            "row_extents": [int(x) for x in vector_literal(b, "rowExtents")],
            "column_count": int(re.search(r"/\*columnCount=\*/(\d+)", b).group(1)),
            "in": vector_literal(b, "rhs"),
            "out_initial": vector_literal(b, "result"),
        }
        m = re.search(r"op\.product\(\s*([-\d.]+),\s*deviceRHS,\s*([-\d.]+),", b)
        case["in_scale"], case["out_scale"] = float(m.group(1)), float(m.group(2))
        case["expected"] = [
            eval(e) for e in re.findall(r"result\[\d\] == Approx\(([^)]*)\)", b)
        ]
        if key == "masked_spmv":
            case["mask"] = [int(x) for x in vector_literal(b, "mask")]
            case["threshold"] = int(re.search(r"threshold = (\d+);", b).group(1))
        out[key] = case
    return out


def stiffness_cases():
    src = read("libraries/fem/packages/integrands/test/LinearIsotropicStiffnessIntegrand_test.cpp")
    basis = re.findall(r"Basis\(\{\s*([-\d.]+),\s*([-\d.]+)\}\)", src)
    modulus = float(re.search(r"modulus = ([-\d.]+);", src).group(1))
    margin = float(re.search(r"\.margin\(([-\deE.]+)\)", src).group(1))
    cases = []
    for m in re.finditer(
        r"references\.emplace_back\(\s*StaticArray<Scalar,Dimension> \{\{([^}]*)\}\},\s*"
        r"std::vector<Scalar> \{\{([^}]*)\}\}",
        src,
    ):
        cases.append({"point": numbers(m.group(1)), "reference": numbers(m.group(2))})
    return {
        "dimension": 2,
        "basis_coefficients": [[float(a), float(b)] for a, b in basis],
        "modulus": modulus,
        "margin": margin,
        "cases": cases,
    }


def gauss_legendre_cases():
    src = read("libraries/fem/packages/numeric/test/GaussLegendreQuadrature_test.cpp")
    tol = float(re.search(r"maxAbsoluteError = ([-\deE.]+);", src).group(1))
    cases = []
    for m in re.finditer(r'CASE_INIT\("order = (\d+)"\)(.*?)GaussLegendreQuadrature<double>', src, re.S):
        order = int(m.group(1))
        vals = numbers(m.group(2).split("reference", 1)[1])
        cases.append({"order": order, "nodes": vals[:order], "weights": vals[order : 2 * order]})
    return {"max_absolute_error": tol, "cases": cases}


def main():
    fixtures = {
        "linalg_space.json": space_cases(),
        "stiffness_integrand.json": stiffness_cases(),
        "gauss_legendre.json": gauss_legendre_cases(),
    }
    for name, data in fixtures.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(data, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    main()
