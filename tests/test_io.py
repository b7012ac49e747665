"""MatrixMarket output: the product's writer against the reference's own
cie::io::MatrixMarket::Output (compiled into oracle/_ref from
cieutils/packages/io/src/MatrixMarket.cpp), byte for byte -- host arrays on the
CPU, the device CSR handle on the GPU."""
import numpy as np
import pytest


def awkward_system():
    """A small CSR matrix whose values exercise the "%g" text: negative zero,
    tiny and huge magnitudes, values that round at the sixth digit, integers,
    Inf and NaN, an empty row, and more columns than rows."""
    rowptr = np.array([0, 3, 3, 7, 10], dtype=np.int32)
    col = np.array([0, 2, 5, 1, 2, 3, 6, 0, 4, 6], dtype=np.int32)
    val = np.array([-0.0, 1e-300, 123456.5, 0.1 + 0.2, -2.5e17, 42.0, 9.999995, np.inf, -np.nan, 1.0 / 3.0])
    return rowptr, col, val


def test_matrix_market_host_writer_matches_reference(tmp_path, reference):
    from cie_b200.fem import make_poisson  # noqa: F401  (package import loads the library)
    from cie_b200.io import write_matrix_market, write_matrix_market_vector
    rp, col, val = awkward_system()
    ours, theirs = tmp_path / "ours.mm", tmp_path / "ref.mm"
    write_matrix_market(ours, (rp, col, val, 7))
    reference.matrix_market(theirs, rp, col, val, columns=7)
    assert ours.read_bytes() == theirs.read_bytes()
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.standard_normal(1000) * 10.0 ** rng.integers(-20, 20, 1000), [0.0, -0.0, np.inf]])
    write_matrix_market_vector(ours, v)
    reference.matrix_market_vector(theirs, v)
    assert ours.read_bytes() == theirs.read_bytes()


def test_matrix_market_large_matches_reference(tmp_path, reference, restatement):
    """A seeded 3D Q1 system (17,576 rows): the chunked parallel formatting writes
    the same bytes as the reference's sequential stream."""
    from cie_b200.io import write_matrix_market
    rp, col, val, b, _, _ = restatement.poisson_system(3, 1, [25, 25, 25], seed=1)
    ours, theirs = tmp_path / "ours.mm", tmp_path / "ref.mm"
    write_matrix_market(ours, (rp, col, val))
    reference.matrix_market(theirs, rp, col, val)
    assert ours.read_bytes() == theirs.read_bytes()


@pytest.mark.gpu
def test_matrix_market_device_matrix_matches_reference(tmp_path, reference):
    import torch
    from cie_b200.fem import make_poisson
    from cie_b200.io import write_matrix_market, write_matrix_market_vector
    from cie_b200.linalg import CUDASpace
    space = CUDASpace()
    prob = make_poisson(space, 2, 2, [20, 20], seed=5)
    ours, theirs = tmp_path / "lhs.mm", tmp_path / "ref.mm"
    write_matrix_market(ours, prob.matrix, space)
    rp, col, val = prob.host_csr()
    reference.matrix_market(theirs, rp, col, val)
    assert ours.read_bytes() == theirs.read_bytes()
    write_matrix_market_vector(ours, prob.rhs, space)
    reference.matrix_market_vector(theirs, prob.rhs.cpu().numpy())
    assert ours.read_bytes() == theirs.read_bytes()
    torch.cuda.synchronize()
