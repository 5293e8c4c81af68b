"""ctypes declarations of the C ABI in include/rsg.h (librsg.so).

Loading fails loudly when the library has not been built; there is no CPU
fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(_HERE)
REPO = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "lib", "librsg.so")
HEADER = os.path.join(REPO, "include", "rsg.h")

# status codes
OK = 0
NOT_CONVERGED = 1
BREAKDOWN = 2
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_OUT_OF_MEMORY = -3
ERR_UNSUPPORTED = -4
ERR_SINGULAR = -5
ERR_TIMEOUT = -6

SOLVER_CG, SOLVER_GMRES = 0, 1
PREC_NONE, PREC_JACOBI, PREC_BLOCK_JACOBI, PREC_LEARNED, PREC_AMG = 0, 1, 2, 3, 4
STOP_REFERENCE, STOP_TRUE_RELRES = 0, 1
PRECISION_FP64, PRECISION_MIXED, PRECISION_AUTO = 0, 1, 2
MEM_HOST, MEM_DEVICE = 0, 1
NOALLOC_MAX_ROWS = 2097152
BC_DISPLACEMENT, BC_DISPLACEMENT_NORMAL, BC_DISPLACEMENT_ROLLER = 1, 2, 4


class SolverConf(C.Structure):
    _fields_ = [
        ("solver_type", C.c_int32),
        ("n_outer", C.c_uint32),
        ("n_inner", C.c_uint32),
        ("cvg", C.c_double),
        ("output_frequency", C.c_uint32),
        ("output_file", C.c_char_p),
        ("eps", C.c_double),
        ("stop_rule", C.c_int32),
        ("rtol", C.c_double),
        ("precision", C.c_int32),
        ("scale_equations", C.c_int32),
        ("reliable_delta", C.c_double),
        ("flexible", C.c_int32),
        ("use_graph", C.c_int32),
        ("check_interval", C.c_uint32),
        ("learned", C.c_void_p),
        ("learned_initial_guess", C.c_int32),
        ("l2_resident_f32", C.c_int32),
        ("autotune", C.c_int32),
        ("amg_sweeps", C.c_int32),
        ("persistent", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32),
        ("outer", C.c_uint32),
        ("error", C.c_double),
        ("trend", C.c_double),
        ("true_relres", C.c_double),
        ("equation_scale", C.c_double),
        ("norm_a", C.c_double),
        ("norm_b", C.c_double),
        ("seconds_setup", C.c_double),
        ("seconds_solve", C.c_double),
        ("converged", C.c_int32),
        ("status", C.c_int32),
        ("fallbacks", C.c_uint32),
        ("fp64_iterations", C.c_uint32),
        ("reserved", C.c_uint32 * 4),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class TuneInfo(C.Structure):
    _fields_ = [
        ("tuned", C.c_int32),
        ("from_cache", C.c_int32),
        ("format", C.c_int32),
        ("rows_per_warp", C.c_uint32),
        ("grid_dir_fp64", C.c_uint32),
        ("grid_dir_fp32", C.c_uint32),
        ("grid_update_fp64", C.c_uint32),
        ("grid_update_fp32", C.c_uint32),
        ("seconds_iter_fp64", C.c_double),
        ("seconds_iter_fp32", C.c_double),
        ("seconds_iter_fp64_default", C.c_double),
        ("seconds_iter_fp32_default", C.c_double),
        ("candidates", C.c_uint32),
        ("pdl_fp64", C.c_int32),
        ("pdl_fp32", C.c_int32),
        ("reserved", C.c_int32 * 1),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ModelGroups(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_uint32),
        ("n_elements", C.c_uint32),
        ("elem_begin", C.c_void_p),
        ("elem_nodes", C.c_void_p),
        ("n_groups", C.c_uint32),
        ("group_begin", C.c_void_p),
        ("group_elems", C.c_void_p),
        ("computable", C.c_void_p),
    ]


class AmgInfo(C.Structure):
    _fields_ = [
        ("levels", C.c_uint32),
        ("dense_coarsest", C.c_uint32),
        ("rows", C.c_uint32 * 16),
        ("nnz", C.c_uint64 * 16),
        ("mis_rounds", C.c_uint32),
        ("setup_launches", C.c_uint32),
        ("seconds_setup", C.c_double),
        ("cycle_launches", C.c_uint32 * 2),
        ("persist_level", C.c_uint32),
    ]


class EigenConf(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("n_eigen", C.c_uint32),
        ("n_iterations", C.c_uint32),
        ("reserved", C.c_uint32),
        ("cvg", C.c_double),
        ("mu0", C.c_double),
    ]


class EigenStats(C.Structure):
    _fields_ = [("n_values", C.c_uint32), ("solves", C.c_uint32), ("iterations", C.c_uint64)]


EIGEN_LANCZOS, EIGEN_ARNOLDI, EIGEN_RAYLEIGH = 0, 1, 2


class Time(C.Structure):
    _fields_ = [("transient", C.c_int32), ("alpha", C.c_double), ("dt", C.c_double)]


_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_U32P = C.POINTER(C.c_uint32)
_U64P = C.POINTER(C.c_uint64)
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "rsg_context_create": (C.c_int, [C.c_int, _PP]),
    "rsg_context_destroy": (None, [_P]),
    "rsg_status_string": (C.c_char_p, [C.c_int]),
    "rsg_last_error": (C.c_char_p, [_P]),
    "rsg_context_set_stream": (C.c_int, [_P, _P]),
    "rsg_synchronize": (C.c_int, [_P]),
    "rsg_conf_default": (None, [C.POINTER(SolverConf)]),
    "rsg_csr_create": (C.c_int, [_P, C.c_uint32, _P, _P, _P, C.c_int32, _PP]),
    "rsg_csr_update_values": (C.c_int, [_P, _P, _P, C.c_int32]),
    "rsg_csr_destroy": (None, [_P, _P]),
    "rsg_csr_info": (C.c_int, [_P, _U32P, _U64P, _DP]),
    "rsg_csr_device_arrays": (C.c_int, [_P, _PP, _PP, _PP]),
    "rsg_csr_copy_to_host": (C.c_int, [_P, _P, _P, _P, _P]),
    "rsg_spmv": (C.c_int, [_P, _P, _P, _P]),
    "rsg_spmv_f32": (C.c_int, [_P, _P, _P, _P]),
    "rsg_jacobi_build": (C.c_int, [_P, _P, _P]),
    "rsg_block_jacobi_build": (C.c_int, [_P, _P, C.c_uint32, _P, _U32P]),
    "rsg_solve": (C.c_int, [_P, _P, C.POINTER(SolverConf), C.c_int32, C.c_uint32, _P, _P, C.c_int32,
                            C.POINTER(Stats)]),
    "rsg_true_relres": (C.c_int, [_P, _P, _P, _P, _DP]),
    "rsg_autotune": (C.c_int, [_P, _P, C.c_char_p, C.POINTER(TuneInfo)]),
    "rsg_csr_save": (C.c_int, [_P, _P, _P, C.c_char_p]),
    "rsg_csr_load": (C.c_int, [_P, C.c_char_p, _PP, _P, _U32P, _U64P, C.POINTER(C.c_int32)]),
    "rsg_selftest_wait_timeout": (C.c_int, [_P, C.c_uint32]),
    "rsg_learned_save": (C.c_int, [_P, _P, C.c_char_p]),
    "rsg_learned_load": (C.c_int, [_P, C.c_char_p, _PP]),
    "rsg_solve_multi": (C.c_int, [_P, _P, C.POINTER(SolverConf), C.c_int32, C.c_uint32, _P, _P, C.c_int32,
                                  C.POINTER(Stats), C.POINTER(Stats)]),
    "rsg_tune_get": (C.c_int, [_P, C.POINTER(TuneInfo)]),
    "rsg_batch_autotune": (C.c_int, [_P, _P, C.POINTER(TuneInfo)]),
    "rsg_profile_kernel": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.c_int32, _DP]),
    "rsg_amg_setup": (C.c_int, [_P, _P, C.POINTER(AmgInfo)]),
    "rsg_amg_setup_conf": (C.c_int, [_P, _P, C.POINTER(SolverConf), C.POINTER(AmgInfo)]),
    "rsg_eigen_solve": (C.c_int, [_P, _P, _P, C.POINTER(EigenConf), C.POINTER(SolverConf), _P, _P, _P,
                                  C.POINTER(EigenStats)]),
    "rsg_amg_level": (C.c_int, [_P, _P, C.c_uint32, _P, _P, _P, _P]),
    "rsg_amg_apply": (C.c_int, [_P, _P, _P, _P, C.c_uint32]),
    "rsg_true_relres_noalloc": (C.c_int, [C.c_uint32, _P, _P, _P, _P, _P, _P, _P]),
    "rsg_batch_create": (C.c_int, [_P, C.c_uint32, _P, _P, _P, _P, _PP]),
    "rsg_batch_destroy": (None, [_P, _P]),
    "rsg_batch_info": (C.c_int, [_P, _U32P, _U32P, _U32P, _U64P]),
    "rsg_batch_solve": (C.c_int, [_P, _P, C.POINTER(SolverConf), C.c_int32, _P, _P, C.c_int32, _P, _P]),
    "rsg_learned_create": (C.c_int, [_P, C.c_uint32, C.c_uint64, _PP]),
    "rsg_learned_destroy": (None, [_P, _P]),
    "rsg_learned_info": (C.c_int, [_P, _U32P, _U32P, _U64P, _U64P]),
    "rsg_learned_get_params": (C.c_int, [_P, _P, _P, C.c_int32]),
    "rsg_learned_set_params": (C.c_int, [_P, _P, _P, C.c_int32]),
    "rsg_learned_set_step": (C.c_int, [_P, C.c_uint64]),
    "rsg_learned_apply": (C.c_int, [_P, _P, _P, _P, _P, _P, C.c_int32]),
    "rsg_learned_loss_grad": (C.c_int, [_P, _P, _P, _P, _P, C.c_int32, _DP]),
    "rsg_learned_train_step": (C.c_int, [_P, _P, _P, _P, _P, C.c_float, _DP]),
    "rsg_node_book_generic": (C.c_int, [C.POINTER(ModelGroups), _P, _P, _U32P]),
    "rsg_node_book_stress": (C.c_int, [C.POINTER(ModelGroups), _P, _P, _P, _U32P]),
    "rsg_assembly_create_heat": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, _P, C.c_uint32, _PP]),
    "rsg_assembly_create_stress": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32, _P, _P, C.c_uint32,
                                             _PP]),
    "rsg_assembly_destroy": (None, [_P, _P]),
    "rsg_assembly_info": (C.c_int, [_P, _U32P, _U64P]),
    "rsg_scatter_plan_create": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, _P, _P, C.c_uint32, _P, C.c_uint32, _PP]),
    "rsg_scatter_plan_info": (C.c_int, [_P, _U64P, _U64P, _U64P]),
    "rsg_scatter_assemble": (C.c_int, [_P, _P, _P, _P, C.c_int32, _PP, _P]),
    "rsg_scatter_plan_destroy": (None, [_P, _P]),
    "rsg_assembly_scatter": (C.c_int, [_P, _P, _P, _P]),
    "rsg_assembly_create_magnetostatics": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, _P, C.c_uint32, _P]),
    "rsg_assemble_magnetostatics": (C.c_int, [_P, _P, _P, _P, C.c_int32, _P, _P]),
    "rsg_assemble_heat": (C.c_int, [_P, _P, _P, _P, _P, _P, C.POINTER(Time), C.c_int32, _PP, _P]),
    "rsg_assemble_stress": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.POINTER(Time), C.c_int32, _PP,
                                      _P]),
}

_lib = None


def header_symbols() -> list[str]:
    """Every function name declared with RSG_API in include/rsg.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"RSG_API\s+[^;(]*?\b(rsg_\w+)\s*\(", txt)))


def load():
    """Load librsg.so, declare every entry point; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not found: build it with `python range-solver-lib_b200/build.py` "
                           "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class RsgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"rsg status {status}: {message}")
        self.status = status
