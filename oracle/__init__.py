"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracle.

* ``port()``: oracle/liboracle.so, the plain-C restatement of the
  reference's hot-path algorithms (la_oracle.c);
* ``ref()``: oracle/_ref/libla_ref.so, the reference's own sources compiled
  in place (ref_shim.cpp + Makefile), or None if it was not built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libla_ref.so"


def reference_tree() -> Path:
    """Where the reference's sources lie: $LA_REFERENCE_TREE if set, else the
    default of oracle/Makefile's REF (the one place that default is kept)."""
    import os
    env = os.environ.get("LA_REFERENCE_TREE")
    if env:
        return Path(env)
    out = subprocess.run(["make", "-s", "-C", str(HERE), "print-ref"], capture_output=True,
                         text=True)
    return Path(out.stdout.strip()) if out.returncode == 0 and out.stdout.strip() else Path()

P, I, D = C.c_void_p, C.c_int, C.c_double

_PORT_SIGS = {
    "oracle_serial_spmv": ([I, I, P, P, P, P, P, D, D], None),
    "oracle_segsum_spmv": ([I, I, I, P, P, P, P, P, D, D], None),
    "oracle_albus_spmv": ([I, I, I, P, P, P, P, P, D, D], None),
    "oracle_segsum_spmv_tiled": ([I, I, I, P, P, P, P, P, D, D], None),
    "oracle_albus_spmv_tiled": ([I, I, I, P, P, P, P, P, D, D], None),
    "oracle_spmv_transpose": ([I, I, I, P, P, P, P, P, D, D], None),
    "oracle_sddmm_pattern": ([I, I, P, P, P, P, P, D], None),
    "oracle_forward_substitution": ([I, I, P, P, P, P, P], None),
    "oracle_forward_substitution_diag": ([I, I, P, P, P, P, P, P], None),
    "oracle_backward_substitution": ([I, I, P, P, P, P, P, P], None),
    "oracle_forward_substitution_t": ([I, I, P, P, P, P, P], None),
    "oracle_level_solve": ([I, P, P, I, P, P, P, P, P, P], None),
    "oracle_level_solve_f32": ([I, P, P, I, P, P, P, P, P, P], None),
    "oracle_topological_sort2": ([I, I, I, P, P, P, P], I),
    "oracle_split_ldu": ([I, I, P, P, P, P, P, P, P, P, P, P, P, P], None),
    "oracle_split_triangle": ([I, I, I, P, P, P, P, P, P], I),
    "oracle_transpose": ([I, I, I, P, P, P, P, P, P], None),
    "oracle_icc0": ([I, I, P, P, P, D, P], I),
    "oracle_rcm": ([I, I, P, P, P, P], None),
    "oracle_permute": ([I, I, P, P, P, P, P, P, P, P], None),
    "oracle_pcg": ([I, I, P, P, P, P, P, P, P, P, D, I, P], I),
}

_REF_SIGS = {
    "la_ref_max_threads": ([], I),
    "la_ref_set_threads": ([I], None),
    "la_ref_serial_spmv": ([I, I, P, P, P, P, P, D, D], None),
    "la_ref_parallel_spmv": ([I, I, I, P, P, P, P, P, D, D], None),
    "la_ref_segsum_create": ([I, I, I, P, P, P], P),
    "la_ref_segsum_apply": ([P, I, I, P, P, P, P, P, D, D], None),
    "la_ref_segsum_destroy": ([P], None),
    "la_ref_albus_create": ([I, I, I, P, P, P], P),
    "la_ref_albus_apply": ([P, I, I, P, P, P, P, P, D, D], None),
    "la_ref_albus_destroy": ([P], None),
    "la_ref_forward_substitution": ([I, I, P, P, P, P, P], None),
    "la_ref_backward_substitution": ([I, I, P, P, P, P, P, P], None),
    "la_ref_forward_substitution_t": ([I, I, P, P, P, P, P], None),
    "la_ref_level_forward": ([I, P, P, I, I, I, P, P, P, P, P], None),
    "la_ref_level_backward": ([I, P, P, I, I, I, P, P, P, P, P, P], None),
    "la_ref_trsv_create": ([I, I, I, I, I, P, P, P, P], P),
    "la_ref_trsv_apply": ([P, P, P], None),
    "la_ref_trsv_destroy": ([P], None),
    "la_ref_topological_sort2": ([I, I, I, P, P, P, P], I),
    "la_ref_topological_sort": ([I, I, I, P, P, P, P], I),
    "la_ref_split_ldu": ([I, I, P, P, P, P, P, P, P, P, P, P, P, P], None),
    "la_ref_split_triangle": ([I, I, I, P, P, P, P, P, P], I),
    "la_ref_transpose": ([I, I, I, P, P, P, P, P, P], None),
    "la_ref_permute": ([I, I, P, P, P, P, P, P, P, P], None),
    "la_ref_valid_csr": ([I, I, I, P, P], I),
    "la_ref_permute_vec": ([I, I, P, P, P], None),
    "la_ref_inverse_permute": ([I, I, P, P], None),
    "la_ref_diagonal": ([I, I, P, P, P, P, P, I], I),
    "la_ref_icc0": ([I, I, P, P, P, D, P], I),
    "la_ref_serial_cm": ([I, I, P, P, P, P], None),
    "la_ref_pcg_create": ([I, I, I, P, P, P, P, P, P], P),
    "la_ref_read_binary_coo": ([C.c_char_p, I, P, P, P, P, P], C.c_longlong),
    "la_ref_read_binary_csr": ([C.c_char_p, I, P, P, P, P, P], C.c_longlong),
    "la_ref_pcg_solve": ([P, P, P, D, I, P], I),
    "la_ref_pcg_destroy": ([P], None),
}

_port = None
_ref = None


def _load(path, sigs):
    L = C.CDLL(str(path))
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


def build(reference_too: bool = True) -> None:
    """Run oracle/Makefile (the C port always; the reference if present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    tree = reference_tree()
    if reference_too and str(tree) not in ("", ".") and (tree / "sparse_mat_op").is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={tree}"], check=True)


def port():
    global _port
    if _port is None:
        if not PORT_SO.exists():
            build(reference_too=False)
        _port = _load(PORT_SO, _PORT_SIGS)
    return _port


def ref():
    global _ref
    if _ref is None and REF_SO.exists():
        _ref = _load(REF_SO, _REF_SIGS)
    return _ref


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
