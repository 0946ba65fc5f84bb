"""ctypes binding of liblab200.so (the C-ABI declared in include/la_b200.h).

The library is loaded from this package directory.  There is no CPU
fallback: if the shared library is missing the import of the binding fails,
and device entry points return LA_ERR_NO_DEVICE without a GPU.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "liblab200.so"

LA_OK = 0
STATUS_NAMES = {
    0: "LA_OK", 1: "LA_ERR_INVALID_ARG", 2: "LA_ERR_BAD_CSR", 3: "LA_ERR_CUDA",
    4: "LA_ERR_TIMEOUT", 5: "LA_ERR_BREAKDOWN", 6: "LA_ERR_NOT_CONVERGED",
    7: "LA_ERR_NO_DEVICE", 8: "LA_ERR_ALLOC",
}
LA_F64, LA_F32 = 0, 1
LA_SPMV_SEGSUM, LA_SPMV_ALBUS = 0, 1
LA_SPMV_MAX_XPARTS = 8  # include/la_b200.h
LA_LOWER, LA_UPPER = 0, 1
LA_CSR_KEEP_F32 = 1
LA_PCG_FP64, LA_PCG_MIXED = 0, 1


class LAError(RuntimeError):
    """A C-ABI call returned a status other than LA_OK."""

    def __init__(self, status: int, func: str, msg: str):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{func}: {self.name}: {msg}")


class PcgInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer_iterations", C.c_int),
                ("rel_residual", C.c_double), ("solve_ms", C.c_double)]


P = C.c_void_p
I = C.c_int
D = C.c_double
IP = C.POINTER(C.c_int)

# name -> argtypes (all return la_status unless listed in _RESTYPES)
_SIGS = {
    "la_last_error_string": [],
    "la_version": [],
    "la_device_sm_count": [IP],
    "la_csr_create": [I, I, I, P, P, P, I, I, C.POINTER(P)],
    "la_csr_create_device": [I, I, I, I, P, P, P, I, I, C.POINTER(P)],
    "la_csr_update_values": [P, P, I],
    "la_csr_download": [P, P, P, P],
    "la_csr_from_coo": [I, I, C.c_longlong, I, P, P, P, I, I, C.POINTER(P)],
    "la_read_binary_coo": [C.c_char_p, I, C.POINTER(C.c_longlong), P, P, P, IP, IP],
    "la_read_matrix_market": [C.c_char_p, C.POINTER(C.c_longlong), P, P, P, IP, IP],
    "la_csr_read_binary_coo": [C.c_char_p, I, I, C.POINTER(P)],
    "la_csr_read_matrix_market": [C.c_char_p, I, C.POINTER(P)],
    "la_csr_parse_matrix_market": [C.c_char_p, C.c_size_t, I, C.POINTER(P)],
    "la_csr_info": [P, IP, IP, IP, IP, IP],
    "la_csr_destroy": [P],
    "la_spmv_plan_create": [P, I, C.POINTER(P)],
    "la_spmv": [P, D, P, D, P, I, P],
    "la_spmv_xparts": [P, D, P, P, I, D, P, I, P],
    "la_spmv_host": [P, D, P, D, P],
    "la_spmv_layout": [P, P],
    "la_spmv_plan_destroy": [P],
    "la_spmv_noalloc": [I, I, I, I, P, P, P, D, P, D, P, P],
    "la_spmv_transpose": [P, D, P, D, P, P],
    "la_sddmm_pattern": [P, D, P, P, P, P],
    "la_topological_sort2": [I, I, I, P, P, P, P, IP],
    "la_rcm": [I, I, P, P, P, P],
    "la_permute": [I, I, P, P, P, P, P, P, P, P],
    "la_transpose": [I, I, I, P, P, P, P, P, P],
    "la_split_ldu": [I, I, P, P, P, P, P, P, P, P, P, P, IP, IP],
    "la_split_triangle": [I, I, I, P, P, P, P, P, P, IP],
    "la_valid_csr": [I, I, I, P, P],
    "la_icc0": [I, I, P, P, P, D, P],
    "la_icc0_shifted": [I, I, P, P, P, P, C.POINTER(C.c_double)],
    "la_trsv_analysis": [I, I, I, P, P, P, P, I, C.POINTER(P)],
    "la_trsv_analysis_levels": [I, I, I, P, P, P, P, I, P, P, I, C.POINTER(P)],
    "la_trsv_analysis_transposed": [I, I, I, P, P, P, P, I, C.POINTER(P)],
    "la_trsv_partition": [I, I, I, P, P, I, P, P],
    "la_trsv_partition_device": [I, I, I, P, P, I, P, P],
    "la_topological_sort": [I, I, I, P, P, P, P, P],
    "la_permute_vec": [I, I, P, P, P],
    "la_ilu0": [I, I, P, P, P, P],
    "la_inverse_permute": [I, I, P, P],
    "la_diagonal": [I, I, P, P, P, P, P, I, P],
    "la_trsv": [P, P, P, P],
    "la_trsv_launch": [P, P, P, P],
    "la_trsv_status": [P, P],
    "la_trsv_host": [P, P, P],
    "la_trsv_levels": [P, IP, P, P],
    "la_trsv_schedule": [P, IP, IP],
    "la_trsv_variant": [P, IP, IP],
    "la_trsv_plan_destroy": [P],
    "la_pcg_create": [P, P, P, P, I, C.POINTER(P)],
    "la_pcg_solve": [P, P, P, D, I, C.POINTER(PcgInfo), P],
    "la_pcg_solve_host": [P, P, P, D, I, C.POINTER(PcgInfo)],
    "la_pcg_adjoint": [P, P, P, P, P, D, I, C.POINTER(PcgInfo), P],
    "la_pcg_fused": [P, IP],
    "la_rcm_device": [I, I, P, P, P, P],
    "la_spmv_ceiling": [P, P, I, P, P],
    "la_topological_sort2_device": [I, I, I, P, P, P, P, IP],
    "la_icc0_plan_create": [I, I, P, P, C.POINTER(P)],
    "la_ilu0_plan_create": [I, I, P, P, C.POINTER(P)],
    "la_factor_numeric": [P, P, D, P, I, IP, P],
    "la_factor_icc0_shifted": [P, P, P, I, C.POINTER(D), P],
    "la_factor_levels": [P, IP],
    "la_factor_plan_destroy": [P],
    "la_pcg_destroy": [P],
}
_RESTYPES = {"la_last_error_string": C.c_char_p, "la_version": C.c_char_p}

_lib = None


def lib() -> C.CDLL:
    """Load liblab200.so once (it must have been built; see build.py)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with "
                "`python -m linearalgebra_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(str(LIB_PATH))
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def last_error() -> str:
    return lib().la_last_error_string().decode(errors="replace")


def call(name: str, *args, ok=(LA_OK,)) -> int:
    """Call a C-ABI function; raise LAError unless the status is in `ok`."""
    st = getattr(lib(), name)(*args)
    if st not in ok:
        raise LAError(st, name, last_error())
    return st


def exported_symbols() -> list[str]:
    return list(_SIGS)
