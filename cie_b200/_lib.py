"""ctypes binding of libciecu.so (the C-ABI in include/ciecu.h, ciecu_host.h,
ciecu_assembly.h).  Loading fails loudly when the library has not been built:
there is no CPU fallback anywhere in this package."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libciecu.so")

c_int, c_int64, c_double, c_float, c_void_p, c_uint16, c_uint64, c_char_p = (
    ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_uint16,
    ctypes.c_uint64, ctypes.c_char_p)
P = c_void_p


class Statistics(ctypes.Structure):
    """IterativeSolver::Statistics (linalg/packages/solvers/inc/IterativeSolver.hpp:21-25)."""
    _fields_ = [("iterationCount", c_int64), ("absoluteResidual", c_double), ("relativeResidual", c_double)]

    def __repr__(self):
        return "Statistics(iterationCount=%d, absoluteResidual=%.6e, relativeResidual=%.6e)" % (
            self.iterationCount, self.absoluteResidual, self.relativeResidual)


class MixedOptions(ctypes.Structure):
    _fields_ = [("mode", c_int), ("delta", c_double), ("compressColumns", c_int), ("innerKernel", c_int),
                ("scaleInner", c_int), ("fuseDirection", c_int)]


class MgOptions(ctypes.Structure):
    _fields_ = [("degree", c_int), ("lambdaMax", c_double), ("ratio", c_double), ("coarseIterations", c_int),
                ("flexible", c_int)]


class MixedStatistics(ctypes.Structure):
    _fields_ = [("iterationCount", c_int64), ("absoluteResidual", c_double), ("relativeResidual", c_double),
                ("innerIterations", c_int64), ("refinements", c_int64), ("trueRelativeResidual", c_double)]


# name -> (restype, argtypes)
SIGNATURES = {
    "ciecu_last_error": (c_int, [c_char_p, c_int]),
    "ciecu_kernel_launch_count": (c_int64, []),
    "ciecu_device_info": (c_int, [P, P, P]),
    "ciecu_space_create": (c_int, [P, P]),
    "ciecu_space_destroy": (c_int, [P]),
    "ciecu_space_synchronize": (c_int, [P]),
    "ciecu_space_stream": (P, [P]),
    "ciecu_alloc": (c_int, [P, ctypes.c_size_t, P]),
    "ciecu_free": (c_int, [P, P]),
    "ciecu_memcpy_h2d": (c_int, [P, P, P, ctypes.c_size_t]),
    "ciecu_memcpy_d2h": (c_int, [P, P, P, ctypes.c_size_t]),
    "ciecu_memcpy_d2d": (c_int, [P, P, P, ctypes.c_size_t]),
    "ciecu_dot_f64": (c_int, [P, c_int64, P, P, P]),
    "ciecu_scale_elementwise_f64": (c_int, [P, c_int64, P, P, c_double]),
    "ciecu_scale_f64": (c_int, [P, c_int64, P, c_double]),
    "ciecu_add_f64": (c_int, [P, c_int64, P, P, c_double]),
    "ciecu_assign_f64": (c_int, [P, c_int64, P, P]),
    "ciecu_fill_f64": (c_int, [P, c_int64, P, c_double]),
    "ciecu_dot_f32": (c_int, [P, c_int64, P, P, P]),
    "ciecu_scale_elementwise_f32": (c_int, [P, c_int64, P, P, c_float]),
    "ciecu_scale_f32": (c_int, [P, c_int64, P, c_float]),
    "ciecu_add_f32": (c_int, [P, c_int64, P, P, c_float]),
    "ciecu_assign_f32": (c_int, [P, c_int64, P, P]),
    "ciecu_fill_f32": (c_int, [P, c_int64, P, c_float]),
    "ciecu_convert_f64_to_f32": (c_int, [P, c_int64, P, P]),
    "ciecu_convert_f32_to_f64": (c_int, [P, c_int64, P, P]),
    "ciecu_csr_create": (c_int, [P, ctypes.c_int32, ctypes.c_int32, c_int64, P, P, P, c_int, P]),
    "ciecu_csr_destroy": (c_int, [P]),
    "ciecu_csr_set_kernel": (c_int, [P, c_int]),
    "ciecu_csr_get_kernel": (c_int, [P, P]),
    "ciecu_csr_diagonals": (c_int, [P, P]),
    "ciecu_csr_autotune": (c_int, [P]),
    "ciecu_csr_spmv_f64": (c_int, [P, c_double, P, c_double, P]),
    "ciecu_csr_spmv_f32": (c_int, [P, c_float, P, c_float, P]),
    "ciecu_csr_masked_spmv_f64": (c_int, [P, P, c_uint16, c_double, P, c_double, P]),
    "ciecu_diagonal_inverse_f64": (c_int, [P, P]),
    "ciecu_diagonal_apply_f64": (c_int, [P, c_int64, P, c_double, P, c_double, P]),
    "ciecu_jacobi_f64": (c_int, [P, P, P, c_uint16, c_int64, c_double, c_double, P, c_double, P, P]),
    "ciecu_jacobi_f64_static": (c_int, [P, P, P, c_uint16, c_int64, c_double, c_double, P, c_double, P]),
    "ciecu_masked_identity_f64": (c_int, [P, c_int64, P, c_uint16, c_double, P, c_double, P]),
    "ciecu_chebyshev_f64": (c_int, [P, P, c_int, c_double, c_double, c_double, P, c_double, P, P]),
    "ciecu_power_lambda_max_f64": (c_int, [P, P, c_int, c_uint64, P, P]),
    "ciecu_pcg_create": (c_int, [P, P, Statistics, c_int, P]),
    "ciecu_pcg_destroy": (c_int, [P]),
    "ciecu_pcg_product": (c_int, [P, c_double, P, c_double, P, P]),
    "ciecu_pcg_set_graph_chunk": (c_int, [P, c_int]),
    "ciecu_pcg_set_schedule": (c_int, [P, c_int]),
    "ciecu_pcg_info": (c_int, [P, P, P]),
    "ciecu_pcg_dia_info": (c_int, [P, P, P]),
    "ciecu_pcg_set_loop": (c_int, [P, c_int]),
    "ciecu_pcg_debug_exchange": (c_int, [P, c_int64, c_int64]),
    "ciecu_mixed_create": (c_int, [P, P, Statistics, MixedOptions, P]),
    "ciecu_mixed_destroy": (c_int, [P]),
    "ciecu_mixed_info": (c_int, [P, P, P]),
    "ciecu_mixed_set_graph_chunk": (c_int, [P, c_int]),
    "ciecu_mixed_product": (c_int, [P, c_double, P, c_double, P, P]),
    "ciecu_mixed_apply_f32": (c_int, [P, P, P]),
    "ciecu_mixed_padded_entries": (c_int, [P, P]),
    "ciecu_mixed_dia_info": (c_int, [P, P, P]),
    "ciecu_mixed_form": (c_int, [P, P]),
    # host utilities
    "ciecu_structured_dofmap": (c_int, [c_int, c_int, P, P, P]),
    "ciecu_structured_boundary": (c_int, [c_int, c_int, P, P]),
    "ciecu_csr_pattern": (c_int, [c_int64, c_int, P, ctypes.c_int32, P, P, P]),
    "ciecu_structured_colors": (c_int, [c_int, P, P]),
    "ciecu_greedy_colors": (c_int, [c_int64, c_int, P, ctypes.c_int32, P, P]),
    "ciecu_random_uniform": (c_int, [c_uint64, c_int64, P]),
    "ciecu_random_normal": (c_int, [c_uint64, c_int64, P]),
    "ciecu_kappa_field": (c_int, [c_uint64, c_int, P, c_double, c_int, P]),
    # assembly
    "ciecu_assembly_create": (c_int, [P, c_int, c_int, c_int, c_int64, P, P, P]),
    "ciecu_assembly_destroy": (c_int, [P]),
    "ciecu_assembly_color_count": (c_int, [P, P]),
    "ciecu_assemble_stiffness": (c_int, [P, P, P, c_int, c_int, P]),
    "ciecu_element_gradient": (c_int, [P, P, c_int, P, P, P, P]),
    "ciecu_adjoint_gradient": (c_int, [P, P, P, c_int, P, P, P, P, P, P, P]),
    "ciecu_assemble_embedded": (c_int, [P, P, P, P, P, P, c_double, c_double, c_int, c_int, c_int, P, P, P]),
    "ciecu_batch_create": (c_int, [P, c_int64, P, P, Statistics, P]),
    "ciecu_batch_destroy": (c_int, [P]),
    "ciecu_batch_info": (c_int, [P, P, P, P]),
    "ciecu_batch_product": (c_int, [P, c_double, P, c_double, P, P]),
    "ciecu_batch_set_refinement": (c_int, [P, c_double]),
    "ciecu_batch_set_reliable_updates": (c_int, [P, c_double]),
    "ciecu_batch_refinements": (c_int, [P, P]),
    "ciecu_multi_create": (c_int, [P, c_int, P, Statistics, P]),
    "ciecu_multi_destroy": (c_int, [P]),
    "ciecu_multi_info": (c_int, [P, P, P]),
    "ciecu_multi_format": (c_int, [P, P]),
    "ciecu_multi_set_format": (c_int, [P, c_int]),
    "ciecu_multi_set_refinement": (c_int, [P, c_double]),
    "ciecu_multi_refinements": (c_int, [P, P]),
    "ciecu_multi_product": (c_int, [P, c_double, P, c_double, P, P]),
    "ciecu_dirichlet_eliminate": (c_int, [P, P, P, P]),
    "ciecu_write_matrix_market_host": (c_int, [c_char_p, c_int64, c_int64, P, P, P]),
    "ciecu_write_matrix_market": (c_int, [P, c_char_p]),
    "ciecu_write_matrix_market_vector": (c_int, [P, c_int64, P, c_char_p]),
    "ciecu_write_matrix_market_vector_host": (c_int, [c_char_p, c_int64, P]),
    "ciecu_make_reordering": (c_int, [P, ctypes.c_int32, P, P, c_int, P]),
    "ciecu_reorder_csr": (c_int, [P, ctypes.c_int32, P, P, P, P, P, P, P]),
    "ciecu_reorder_vector": (c_int, [P, c_int64, P, c_int, P, P]),
    "ciecu_csr_pattern_device": (c_int, [P, c_int64, c_int, P, ctypes.c_int32, P, P, P]),
    "ciecu_assemble_dirichlet_penalty": (c_int, [P, P, P, c_double, c_int, c_int, P, P, P]),
    "ciecu_assemble_embedded_f32": (c_int, [P, P, P, P, P, P, c_double, c_double, c_int, c_int, c_int, P, P]),
    "ciecu_dirichlet_eliminate_f32": (c_int, [P, P, P]),
    "ciecu_mgcg_create": (c_int, [P, P, P, P, P, P, P, MgOptions, Statistics, P]),
    "ciecu_mgcg_destroy": (c_int, [P]),
    "ciecu_mgcg_product": (c_int, [P, c_double, P, c_double, P, P]),
    "ciecu_mgcg_info": (c_int, [P, P, P]),
    "ciecu_mgcg_smoother_info": (c_int, [P, P, P]),
    "ciecu_mgcg_coarse_info": (c_int, [P, P, P]),
    "ciecu_mgcg_set_coarse_cluster": (c_int, [P, c_int]),
    "ciecu_mgcg_coarse_apply": (c_int, [P, P, P]),
}

OPTIONAL = set()

STATUS_NAMES = {1: "ARGUMENT", 2: "CUDA", 3: "BREAKDOWN", 4: "DIAGONAL", 5: "TIMEOUT", 6: "PATTERN"}


class CiecuError(RuntimeError):
    """Non-zero status of a ciecu_* call (the C++ wrapper raises cie::Exception)."""

    def __init__(self, status, message):
        super().__init__("%s (ciecu status %d %s)" % (message, status, STATUS_NAMES.get(status, "?")))
        self.status = status


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("cie_b200: %s is missing; build it with `python -m cie_b200.build` "
                          "(there is no CPU fallback)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        try:
            f = getattr(lib, name)
        except AttributeError:
            if name in OPTIONAL:
                continue
            raise
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error():
    buf = ctypes.create_string_buffer(4096)
    load().ciecu_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status):
    if status != 0:
        raise CiecuError(status, last_error())
    return status


def call(name, *args):
    return check(getattr(load(), name)(*args))
