"""Python mirror of the reference's hot-path interface over the C-ABI.

Names, argument order and meaning follow the reference's C++ API
(sparse_mat_op/spmv.hpp, triangle_solve.hpp, matrix_utils.hpp,
precond.hpp, reordering/Reordering.cpp):

* ``SegSumSPMV`` / ``ALBUSSPMV``: ``preprocess(size, base, ai, aj, av)`` then
  ``spmv(size, base, ai, aj, av, b, x, alpha, beta)`` computing
  x = alpha*A*b + beta*x (spmv.hpp:68-82, 195-233).  ``preprocess`` uploads
  the matrix and builds the tile plan once; later calls must pass the same
  matrix (as the reference's preprocessed state assumes).  ``b`` / ``x`` may
  be numpy arrays (host path: copied in and out) or CUDA torch tensors
  (device path, on the current stream).
* ``SPMV(csr, kind)``: the ``SPMV<CSR, Impl>`` adapter (spmv.hpp:310-334).
* ``OptimizedTriangularSolve(uplo)``: ``analysis(rows, base, ai, aj, av,
  diag=None)`` then ``solve(b, x)`` (triangle_solve.hpp:149-171).
* ``TopologicalSort2``, ``SplitLDU``, ``SplitTriangle``, ``Transpose``,
  ``Permute``, ``ValidCSR``, ``ICCLevelNumeric0``, ``SerialCM``: the host
  preprocessing steps, bit-identical to the reference's.
* ``PCG``: IC(0)-preconditioned CG (FP64 or mixed precision).

Everything computes on the GPU through liblab200.so; nothing falls back to
the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (LA_CSR_KEEP_F32, LA_F32, LA_F64, LA_LOWER, LA_PCG_FP64,
                   LA_PCG_MIXED, LA_SPMV_ALBUS, LA_SPMV_MAX_XPARTS, LA_SPMV_SEGSUM, LA_UPPER,
                   LAError, PcgInfo, call)

__all__ = [
    "CSR", "SPMV", "SegSumSPMV", "ALBUSSPMV", "OptimizedTriangularSolve",
    "TopologicalSort2", "SplitLDU", "SplitTriangle", "Transpose", "Permute",
    "ValidCSR", "ICCLevelNumeric0", "ICCShifted", "SerialCM", "PCG", "LAError",
    "spmv_transpose", "sddmm_pattern", "ForwardSubstitutionT", "ForwardSubstitution",
    "BackwardSubstitution", "LevelScheduleForwardSubstitution",
    "LevelScheduleBackwardSubstitution", "trsv_partition", "TopologicalSort",
    "PermuteVec", "InversePermute", "Diagonal", "ILU0", "csr_from_coo", "ReadFromBinaryCOO",
    "read_matrix_market_coo", "ReadFromBinaryCSR", "read_matrix_market_csr", "FactorPlan",
]


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a) -> C.c_void_p:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())  # torch tensor


def _stream(t) -> C.c_void_p:
    import torch
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _release(fn: str, obj) -> None:
    """Destroy a handle; quiet during interpreter shutdown."""
    h = getattr(obj, "h", None)
    obj.h = None
    if h is not None and h.value:
        try:
            getattr(_lib.lib(), fn)(h)
        except Exception:
            pass


def _is_device(a) -> bool:
    return not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


# ------------------------------------------------------------------ CSR
class CSR:
    """Device copy of a CSR matrix (host arrays are validated and copied)."""

    def __init__(self, n, ncols, base, ai, aj, av, dtype=np.float64,
                 keep_f32=False):
        ai, aj = _i32(ai), _i32(aj)
        av = np.ascontiguousarray(av, dtype=dtype)
        self.n, self.ncols, self.base = int(n), int(ncols), int(base)
        self.nnz = int(ai[n] - base)
        self.dtype = np.dtype(dtype)
        h = C.c_void_p()
        call("la_csr_create", self.n, self.ncols, self.base, _ptr(ai), _ptr(aj),
             _ptr(av), LA_F64 if self.dtype == np.float64 else LA_F32,
             LA_CSR_KEEP_F32 if keep_f32 else 0, C.byref(h))
        self.h = h
        self.host = (ai, aj, av)

    @classmethod
    def _adopt(cls, h, keep_host=True):
        """Wrap a handle the library created (ingest); host arrays downloaded."""
        self = cls.__new__(cls)
        self.h = h
        n, nc, nnz, base, dt = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        call("la_csr_info", h, C.byref(n), C.byref(nc), C.byref(nnz), C.byref(base),
             C.byref(dt))
        self.n, self.ncols, self.nnz, self.base = n.value, nc.value, nnz.value, base.value
        self.dtype = np.dtype(np.float64 if dt.value == LA_F64 else np.float32)
        self.host = self.download() if keep_host else None
        return self

    def download(self):
        """(ai, aj, av) host copies of the device arrays (la_csr_download)."""
        ai = np.empty(self.n + 1, np.int32)
        aj = np.empty(self.nnz, np.int32)
        av = np.empty(self.nnz, self.dtype)
        call("la_csr_download", self.h, _ptr(ai), _ptr(aj), _ptr(av))
        return ai, aj, av

    def update_values(self, av):
        if _is_device(av):
            call("la_csr_update_values", self.h, _ptr(av), 1)
        else:
            av = np.ascontiguousarray(av, dtype=self.dtype)
            call("la_csr_update_values", self.h, _ptr(av), 0)

    def __del__(self):
        _release("la_csr_destroy", self)


class SPMV:
    """``SPMV<CSR, Impl>`` (spmv.hpp:310-334): y = alpha*A*x + beta*y."""

    def __init__(self, A: CSR, kind: int = LA_SPMV_SEGSUM):
        self.A = A
        h = C.c_void_p()
        call("la_spmv_plan_create", A.h, int(kind), C.byref(h))
        self.h = h

    def __call__(self, b, x, alpha=1.0, beta=0.0):
        """x = alpha*A*b + beta*x; b/x numpy (host path) or CUDA tensors."""
        if _is_device(b):
            import torch
            vd = LA_F64 if b.dtype == torch.float64 else LA_F32
            call("la_spmv", self.h, float(alpha), _ptr(b), float(beta), _ptr(x),
                 vd, _stream(b))
        else:
            if not (isinstance(x, np.ndarray) and x.dtype == np.float64
                    and x.flags.c_contiguous):
                raise TypeError("host x must be a C-contiguous float64 array")
            b = _f64(b)
            call("la_spmv_host", self.h, float(alpha), _ptr(b), float(beta),
                 _ptr(x))
        return x

    def layout(self):
        """0 for the tile pass, k > 0 for the row-slot form with k slots a row
        (la_spmv_layout)."""
        k = C.c_int()
        call("la_spmv_layout", self.h, C.byref(k))
        return k.value

    def xparts(self, slices, starts, y, alpha=1.0, beta=0.0):
        """y = alpha*A*x + beta*y with x given as contiguous slices: slices[r]
        holds columns starts[r]..starts[r+1]-1; each entry is a CUDA tensor or a
        raw device address (e.g. a peer GPU's buffer).  la_spmv_xparts."""
        import torch
        ptrs = (C.c_void_p * len(slices))(
            *[s if isinstance(s, int) else s.data_ptr() for s in slices])
        st = np.ascontiguousarray(starts, dtype=np.int32)
        vd = LA_F64 if y.dtype == torch.float64 else LA_F32
        call("la_spmv_xparts", self.h, float(alpha), C.cast(ptrs, C.c_void_p), _ptr(st),
             len(slices), float(beta), _ptr(y), vd, _stream(y))
        return y

    def ceiling(self, x, gather=True, sink=None):
        """The matrix's streaming bound for the tile pass (la_spmv_ceiling):
        its columns and values streamed, x gathered when ``gather``; a
        measurement aid, not an SpMV."""
        import torch
        if sink is None:
            sink = torch.zeros(1, dtype=torch.float64, device=x.device)
        call("la_spmv_ceiling", self.h, _ptr(x), int(bool(gather)), _ptr(sink), _stream(x))
        return sink

    def transpose(self, g, out, alpha=1.0, beta=0.0):
        """out = alpha*A^T g + beta*out (device FP64 tensors)."""
        call("la_spmv_transpose", self.h, float(alpha), _ptr(g), float(beta),
             _ptr(out), _stream(g))
        return out

    def sddmm(self, g, x, dv, alpha=1.0):
        """dv[k] = alpha*g[row(k)]*x[col(k)] (device FP64 tensors)."""
        call("la_sddmm_pattern", self.h, float(alpha), _ptr(g), _ptr(x),
             _ptr(dv), _stream(g))
        return dv

    def __del__(self):
        _release("la_spmv_plan_destroy", self)


def spmv_transpose(plan: SPMV, g, out, alpha=1.0, beta=0.0):
    return plan.transpose(g, out, alpha, beta)


def sddmm_pattern(plan: SPMV, g, x, dv, alpha=1.0):
    return plan.sddmm(g, x, dv, alpha)


class SegSumSPMV:
    """``SegSumSPMV`` (spmv.hpp:59-185) on the GPU."""

    KIND = LA_SPMV_SEGSUM

    def __init__(self, num_threads: int | None = None):
        self._nthreads = num_threads  # kept for API parity; the GPU ignores it
        self._plan = None
        self._key = None

    def setNumThreads(self, num_threads: int):
        self._nthreads = num_threads

    def preprocess(self, size, base, ai, aj, av):
        ai, aj, av = _i32(ai), _i32(aj), _f64(av)
        ncols = int(aj.max()) + 1 - base if aj.size else size
        ncols = max(ncols, size)
        self._A = CSR(size, ncols, base, ai, aj, av)
        self._plan = SPMV(self._A, self.KIND)
        self._key = (int(size), int(base))

    def __call__(self, size, base, ai, aj, av, b, x, alpha=1.0, beta=0.0):
        if self._plan is None or self._key != (int(size), int(base)):
            self.preprocess(size, base, ai, aj, av)
        return self._plan(b, x, alpha, beta)


class ALBUSSPMV(SegSumSPMV):
    """``ALBUSSPMV`` (spmv.hpp:186-300) on the GPU."""

    KIND = LA_SPMV_ALBUS


# ------------------------------------------------- device factorisation
class FactorPlan:
    """IC(0) or ILU(0) on the GPU, bit-identical to ``ICCLevelNumeric0`` /
    ``ILU0``: the pattern is analysed once (``kind`` "ic0": u_ai/u_aj the
    upper triangle with diagonals first; "ilu0": a full pattern), then
    ``factor`` runs numeric passes on the device."""

    def __init__(self, kind, n, base, ai, aj):
        ai, aj = _i32(ai), _i32(aj)
        self.kind, self.n, self.nnz = kind, int(n), int(ai[n] - base)
        h = C.c_void_p()
        fn = {"ic0": "la_icc0_plan_create", "ilu0": "la_ilu0_plan_create"}[kind]
        call(fn, int(n), int(base), _ptr(ai), _ptr(aj), C.byref(h))
        self.h = h

    def factor(self, av, omega=0.0, out=None):
        """The factor of values av (host array -> numpy result; CUDA tensor
        -> written into `out`, a CUDA tensor).  LAError LA_ERR_BREAKDOWN on
        a negative IC / zero ILU pivot; its ``bad_row`` is the first such
        row."""
        bad = C.c_int(-1)
        if _is_device(av):
            st = call("la_factor_numeric", self.h, _ptr(av), float(omega), _ptr(out), 1,
                      C.byref(bad), _stream(av), ok=(0, 5))
            res = out
        else:
            av = _f64(av)
            res = np.empty(self.nnz)
            st = call("la_factor_numeric", self.h, _ptr(av), float(omega), _ptr(res), 0,
                      C.byref(bad), None, ok=(0, 5))
        if st == 5:
            e = LAError(st, "la_factor_numeric", _lib.last_error())
            e.bad_row = bad.value
            raise e
        return res

    def shifted(self, av):
        """IC(0) with the reference's shift retries: (factor, shift used)."""
        av = _f64(av)
        res = np.empty(self.nnz)
        sh = C.c_double()
        call("la_factor_icc0_shifted", self.h, _ptr(av), _ptr(res), 0, C.byref(sh), None)
        return res, sh.value

    def levels(self):
        lv = C.c_int()
        call("la_factor_levels", self.h, C.byref(lv))
        return lv.value

    def __del__(self):
        _release("la_factor_plan_destroy", self)


# --------------------------------------------------------------- ingest
def csr_from_coo(nrows, ncols, base, rows, cols, vals, dtype=np.float64, keep_f32=False):
    """Device CSR from host COO entries (indices carry `base`), ordered by
    (row, col) on the device; equal (row, col) entries kept in input order."""
    rows, cols = _i32(rows), _i32(cols)
    vals = np.ascontiguousarray(vals, dtype=dtype)
    h = C.c_void_p()
    call("la_csr_from_coo", int(nrows), int(ncols), len(rows), int(base), _ptr(rows),
         _ptr(cols), _ptr(vals), LA_F64 if np.dtype(dtype) == np.float64 else LA_F32,
         LA_CSR_KEEP_F32 if keep_f32 else 0, C.byref(h))
    return CSR._adopt(h)


def _two_call(fn, *lead):
    nnz, m, n = C.c_longlong(), C.c_int(), C.c_int()
    call(fn, *lead, C.byref(nnz), None, None, None, C.byref(m), C.byref(n))
    rows, cols = np.empty(nnz.value, np.int32), np.empty(nnz.value, np.int32)
    vals = np.empty(nnz.value, np.float64)
    call(fn, *lead, C.byref(nnz), _ptr(rows), _ptr(cols), _ptr(vals), C.byref(m), C.byref(n))
    return m.value, n.value, rows, cols, vals


def ReadFromBinaryCOO(filename, base=0):
    """``utils::ReadFromBinaryCOO`` (utils/utils.h:23-44), host:
    (rows, cols, vals, (m, n)) in file order."""
    m, n, r, c, v = _two_call("la_read_binary_coo", str(filename).encode(), int(base))
    return r, c, v, (m, n)


def read_matrix_market_coo(filename):
    """0-based COO entries of a Matrix Market coordinate file, symmetric
    storage expanded: (m, n, rows, cols, vals)."""
    return _two_call("la_read_matrix_market", str(filename).encode())


def ReadFromBinaryCSR(filename, base=0, keep_f32=False):
    """``utils::ReadFromBinaryCSR`` (utils/utils.h:46-91) into a device CSR
    (the file's base); ``.host`` holds (ai, aj, av)."""
    h = C.c_void_p()
    call("la_csr_read_binary_coo", str(filename).encode(), int(base),
         LA_CSR_KEEP_F32 if keep_f32 else 0, C.byref(h))
    return CSR._adopt(h)


def read_matrix_market_csr(filename, keep_f32=False):
    """``utils::read_matrix_market_csr`` (utils/utils.h:93-132) into a
    0-based device CSR; ``.host`` holds (ai, aj, av)."""
    h = C.c_void_p()
    call("la_csr_read_matrix_market", str(filename).encode(),
         LA_CSR_KEEP_F32 if keep_f32 else 0, C.byref(h))
    return CSR._adopt(h)


# ----------------------------------------------------------- triangular
class OptimizedTriangularSolve:
    """``OptimizedTriangularSolve<Barrier, L|U>`` (triangle_solve.hpp:149-208)."""

    def __init__(self, uplo: str = "L", num_threads: int | None = None,
                 dtype=np.float64):
        self.uplo = LA_LOWER if uplo in ("L", 0, LA_LOWER) else LA_UPPER
        self._nthreads = num_threads
        self.dtype = np.dtype(dtype)
        self.h = None

    def analysis(self, rows, base, ai, aj, av, diag=None):
        ai, aj, av = _i32(ai), _i32(aj), _f64(av)
        d = None if diag is None else _f64(diag)
        h = C.c_void_p()
        call("la_trsv_analysis", self.uplo, int(rows), int(base), _ptr(ai),
             _ptr(aj), _ptr(av), _ptr(d),
             LA_F64 if self.dtype == np.float64 else LA_F32, C.byref(h))
        self.h = h
        self.n = int(rows)
        return self

    def analysis_transposed(self, rows, base, ai, aj, av, diag=None):
        """Plan the solve with T^T, given the CSR of the strict triangle T of
        the other kind (strict U for an "L" solver); the role
        ForwardSubstitutionT (triangle_solve.hpp:87-98) plays."""
        ai, aj, av = _i32(ai), _i32(aj), _f64(av)
        d = None if diag is None else _f64(diag)
        h = C.c_void_p()
        t_uplo = LA_UPPER if self.uplo == LA_LOWER else LA_LOWER
        call("la_trsv_analysis_transposed", t_uplo, int(rows), int(base), _ptr(ai),
             _ptr(aj), _ptr(av), _ptr(d),
             LA_F64 if self.dtype == np.float64 else LA_F32, C.byref(h))
        self.h = h
        self.n = int(rows)
        return self

    def analysis_levels(self, rows, base, ai, aj, av, iperm, prefix, diag=None):
        """analysis() with a caller-built level structure (iperm, prefix)."""
        ai, aj, av = _i32(ai), _i32(aj), _f64(av)
        iperm, prefix = _i32(iperm), _i32(prefix)
        d = None if diag is None else _f64(diag)
        h = C.c_void_p()
        call("la_trsv_analysis_levels", self.uplo, int(rows), int(base), _ptr(ai),
             _ptr(aj), _ptr(av), _ptr(d),
             LA_F64 if self.dtype == np.float64 else LA_F32, _ptr(iperm),
             _ptr(prefix), len(prefix) - 1, C.byref(h))
        self.h = h
        self.n = int(rows)
        return self

    def schedule(self):
        """('levels', 0), ('parts', number of parts) or ('parts-ring', number of
        parts): the analysis's choice."""
        s, p = C.c_int(), C.c_int()
        call("la_trsv_schedule", self.h, C.byref(s), C.byref(p))
        return {0: "levels", 1: "parts", 2: "parts-ring"}[s.value], p.value

    def variant(self):
        """(register slots per row, second-row register sets): the kernel
        variant the analysis picked (la_trsv_variant)."""
        k, w = C.c_int(), C.c_int()
        call("la_trsv_variant", self.h, C.byref(k), C.byref(w))
        return k.value, bool(w.value)

    def levels(self):
        lv = C.c_int()
        call("la_trsv_levels", self.h, C.byref(lv), None, None)
        iperm = np.empty(self.n, np.int32)
        prefix = np.empty(lv.value + 1, np.int32)
        call("la_trsv_levels", self.h, C.byref(lv), _ptr(iperm), _ptr(prefix))
        return lv.value, iperm, prefix

    def __call__(self, b, x):
        if _is_device(b):
            call("la_trsv", self.h, _ptr(b), _ptr(x), _stream(b))
        else:
            b = _f64(b)
            call("la_trsv_host", self.h, _ptr(b), _ptr(x))
        return x

    def launch(self, b, x):
        """Asynchronous device solve; errors surface in status()."""
        call("la_trsv_launch", self.h, _ptr(b), _ptr(x), _stream(b))
        return x

    def status(self, t):
        call("la_trsv_status", self.h, _stream(t))

    def get_num_threads(self):
        return self._nthreads

    def __del__(self):
        _release("la_trsv_plan_destroy", self)


# --------------------------------------------------------- host analysis
def trsv_partition(uplo, n, base, ai, aj, nparts, device=False):
    """(part[n], coordinates used): the row partition the partitioned solve
    schedule cuts for this strict triangle -- on the host, or with its
    landmark stage on the GPU (``device=True``, as the analysis computes it;
    the same partition)."""
    ai, aj = _i32(ai), _i32(aj)
    part = np.empty(max(n, 1), np.int32)
    c = C.c_int()
    call("la_trsv_partition_device" if device else "la_trsv_partition",
         LA_LOWER if uplo in ("L", 0, LA_LOWER) else LA_UPPER, int(n),
         int(base), _ptr(ai), _ptr(aj), int(nparts), _ptr(part), C.byref(c))
    return part[:n], c.value


def ForwardSubstitution(size, base, ai, aj, av, b, x):
    """``ForwardSubstitution`` (triangle_solve.hpp:32-43): unit lower solve with
    the strict lower CSR, host arrays, x written in place (one GPU plan and
    solve per call; keep an OptimizedTriangularSolve for repeated solves)."""
    OptimizedTriangularSolve("L").analysis(size, base, ai, aj, av)(_f64(b), x)
    return x


def BackwardSubstitution(size, base, ai, aj, av, diag, b, x):
    """``BackwardSubstitution`` (triangle_solve.hpp:59-71): strict upper CSR
    plus diag, host arrays, x written in place."""
    OptimizedTriangularSolve("U").analysis(size, base, ai, aj, av, diag)(_f64(b), x)
    return x


def LevelScheduleForwardSubstitution(iperm, prefix, lvls, rows, base, ai, aj, av, b, x):
    """``LevelScheduleForwardSubstitution`` (triangle_solve.hpp:100-122) with the
    caller's levels (iperm with base, zero-based prefix[lvls + 1])."""
    OptimizedTriangularSolve("L").analysis_levels(
        rows, base, ai, aj, av, iperm, _i32(prefix)[:int(lvls) + 1])(_f64(b), x)
    return x


def LevelScheduleBackwardSubstitution(iperm, prefix, lvls, rows, base, ai, aj, av, diag, b, x):
    """``LevelScheduleBackwardSubstitution`` (triangle_solve.hpp:124-145)."""
    OptimizedTriangularSolve("U").analysis_levels(
        rows, base, ai, aj, av, iperm, _i32(prefix)[:int(lvls) + 1], diag)(_f64(b), x)
    return x


def ForwardSubstitutionT(size, base, ai, aj, av, b, x):
    """``ForwardSubstitutionT`` (triangle_solve.hpp:87-98): x = (I + U^T)^-1 b
    for the strict upper triangle U given as CSR; host arrays, x written in
    place.  Plans the transposed solve on the GPU and runs it once."""
    ts = OptimizedTriangularSolve("L").analysis_transposed(size, base, ai, aj, av)
    ts(np.ascontiguousarray(b, np.float64), x)
    return x


def TopologicalSort(uplo, nodes, base, ai, aj):
    """``TopologicalSort`` (matrix_utils.hpp:583-635, Kahn's order): returns
    (the reference's return value = last level index, iperm, prefix)."""
    ai, aj = _i32(ai), _i32(aj)
    iperm = np.empty(max(nodes, 1), np.int32)
    prefix = np.empty(nodes + 2, np.int32)
    r = C.c_int()
    call("la_topological_sort", LA_LOWER if uplo in ("L", 0) else LA_UPPER, int(nodes),
         int(base), _ptr(ai), _ptr(aj), _ptr(iperm), _ptr(prefix), C.byref(r))
    return r.value, iperm[:nodes], prefix[: r.value + 2].copy()


def TopologicalSort2(uplo, nodes, base, ai, aj, device=False):
    """Level sets (matrix_utils.hpp:637-675): returns (levels, iperm, prefix);
    ``device=True`` computes them on the GPU (la_topological_sort2_device,
    same outputs; strict triangles only)."""
    ai, aj = _i32(ai), _i32(aj)
    iperm = np.empty(nodes, np.int32)
    prefix = np.empty(nodes + 1, np.int32)
    lv = C.c_int()
    call("la_topological_sort2_device" if device else "la_topological_sort2",
         LA_LOWER if uplo in ("L", 0) else LA_UPPER,
         int(nodes), int(base), _ptr(ai), _ptr(aj), _ptr(iperm), _ptr(prefix),
         C.byref(lv))
    return lv.value, iperm, prefix[: lv.value + 1].copy()


def SerialCM(n, base, ai, aj, device=False):
    """Reverse Cuthill-McKee (reordering/Reordering.cpp:37-136): (iperm, perm);
    ``device=True`` orders large components on the GPU (la_rcm_device, the
    same ordering)."""
    ai, aj = _i32(ai), _i32(aj)
    iperm = np.empty(n, np.int32)
    perm = np.empty(n, np.int32)
    call("la_rcm_device" if device else "la_rcm", int(n), int(base), _ptr(ai), _ptr(aj),
         _ptr(iperm), _ptr(perm))
    return iperm, perm


def Permute(n, base, ai, aj, av, iperm, perm=None):
    """matrix_utils.hpp:429-480: B(i,:) = A(iperm[i],:), columns via perm."""
    ai, aj, av, iperm = _i32(ai), _i32(aj), _f64(av), _i32(iperm)
    perm = None if perm is None else _i32(perm)
    nnz = int(ai[n] - base)
    p_ai = np.empty(n + 1, np.int32)
    p_aj = np.empty(max(nnz, 1), np.int32)
    p_av = np.empty(max(nnz, 1), np.float64)
    call("la_permute", int(n), int(base), _ptr(ai), _ptr(aj), _ptr(av),
         _ptr(iperm), _ptr(perm), _ptr(p_ai), _ptr(p_aj), _ptr(p_av))
    return p_ai, p_aj[:nnz], p_av[:nnz]


def ILU0(n, base, ai, aj, av):
    """ILU(0) on A's pattern (host): L strictly below the diagonal (unit
    diagonal implied) and U on and above it, in A's pattern."""
    ai, aj, av = _i32(ai), _i32(aj), _f64(av)
    lu = np.empty(max(len(av), 1), np.float64)
    call("la_ilu0", int(n), int(base), _ptr(ai), _ptr(aj), _ptr(av), _ptr(lu))
    return lu[: len(av)]


def PermuteVec(rows, base, v, iperm=None):
    """``permuteVec`` (matrix_utils.hpp:562-576): v[iperm[i] - base]."""
    v = _f64(v)
    out = np.empty(rows, np.float64)
    ip = None if iperm is None else _i32(iperm)
    call("la_permute_vec", int(rows), int(base), _ptr(v), _ptr(ip), _ptr(out))
    return out


def InversePermute(perm, base=0):
    """``inversePermute`` (utils.cpp:101-108): iperm[perm[i] - base] = i + base."""
    perm = _i32(perm)
    iperm = np.empty(len(perm), np.int32)
    call("la_inverse_permute", len(perm), int(base), _ptr(perm), _ptr(iperm))
    return iperm


def Diagonal(rows, base, ai, aj, av, invert=False):
    """``Diagonal`` (matrix_utils.hpp:677-704): (all diagonal entries present,
    diagpos with base, diag values)."""
    ai, aj, av = _i32(ai), _i32(aj), _f64(av)
    pos = np.empty(rows, np.int32)
    d = np.empty(rows, np.float64)
    ok = C.c_int()
    call("la_diagonal", int(rows), int(base), _ptr(ai), _ptr(aj), _ptr(av), _ptr(pos),
         _ptr(d), 1 if invert else 0, C.byref(ok))
    return bool(ok.value), pos, d


def Transpose(rows, cols, base, ai, aj, av=None):
    """ParallelTranspose2 (matrix_utils.hpp:311-390)."""
    ai, aj = _i32(ai), _i32(aj)
    avp = None if av is None else _f64(av)
    nnz = int(ai[rows] - base)
    t_ai = np.empty(cols + 1, np.int32)
    t_aj = np.empty(max(nnz, 1), np.int32)
    t_av = None if av is None else np.empty(max(nnz, 1), np.float64)
    call("la_transpose", int(rows), int(cols), int(base), _ptr(ai), _ptr(aj),
         _ptr(avp), _ptr(t_ai), _ptr(t_aj), _ptr(t_av))
    return t_ai, t_aj[:nnz], (None if t_av is None else t_av[:nnz])


def SplitLDU(n, base, ai, aj, av):
    """SplitLDU (matrix_utils.hpp:720-803): ((L), D, (U)) as CSR triples."""
    ai, aj, av = _i32(ai), _i32(aj), _f64(av)
    nnz = max(int(ai[n] - base), 1)
    l_ai, u_ai = np.empty(n + 1, np.int32), np.empty(n + 1, np.int32)
    l_aj, u_aj = np.empty(nnz, np.int32), np.empty(nnz, np.int32)
    l_av, u_av = np.empty(nnz, np.float64), np.empty(nnz, np.float64)
    d = np.empty(n, np.float64)
    ln, un = C.c_int(), C.c_int()
    call("la_split_ldu", int(n), int(base), _ptr(ai), _ptr(aj), _ptr(av),
         _ptr(l_ai), _ptr(l_aj), _ptr(l_av), _ptr(d), _ptr(u_ai), _ptr(u_aj),
         _ptr(u_av), C.byref(ln), C.byref(un))
    return ((l_ai, l_aj[: ln.value].copy(), l_av[: ln.value].copy()), d,
            (u_ai, u_aj[: un.value].copy(), u_av[: un.value].copy()))


def SplitTriangle(uplo, n, base, ai, aj, av):
    """SplitTriangle<L|U> (matrix_utils.hpp:805-879), diagonal included."""
    ai, aj, av = _i32(ai), _i32(aj), _f64(av)
    nnz = max(int(ai[n] - base), 1)
    t_ai, t_aj, t_av = (np.empty(n + 1, np.int32), np.empty(nnz, np.int32),
                        np.empty(nnz, np.float64))
    tn = C.c_int()
    call("la_split_triangle", LA_LOWER if uplo in ("L", 0) else LA_UPPER,
         int(n), int(base), _ptr(ai), _ptr(aj), _ptr(av), _ptr(t_ai),
         _ptr(t_aj), _ptr(t_av), C.byref(tn))
    return t_ai, t_aj[: tn.value].copy(), t_av[: tn.value].copy()


def ValidCSR(rows, cols, base, ai, aj) -> bool:
    """ValidCSR (matrix_utils.hpp:985-1014)."""
    ai, aj = _i32(ai), _i32(aj)
    st = call("la_valid_csr", int(rows), int(cols), int(base), _ptr(ai),
              _ptr(aj), ok=(0, 2))
    return st == 0


def ICCLevelNumeric0(n, base, u_ai, u_aj, u_av, omega=0.0):
    """IC(0) factor (precond.hpp:13-37, 615-693) of the upper triangle.

    Returns the factor values; raises LAError(LA_ERR_BREAKDOWN) on a
    negative pivot, the reference's ``false`` return.
    """
    u_ai, u_aj, u_av = _i32(u_ai), _i32(u_aj), _f64(u_av)
    out = np.empty_like(u_av)
    call("la_icc0", int(n), int(base), _ptr(u_ai), _ptr(u_aj), _ptr(u_av),
         float(omega), _ptr(out))
    return out


def ICCShifted(n, base, u_ai, u_aj, u_av):
    """IC(0) with the reference's shift-retry loop; returns (values, shift)."""
    u_ai, u_aj, u_av = _i32(u_ai), _i32(u_aj), _f64(u_av)
    out = np.empty_like(u_av)
    sh = C.c_double()
    call("la_icc0_shifted", int(n), int(base), _ptr(u_ai), _ptr(u_aj),
         _ptr(u_av), _ptr(out), C.byref(sh))
    return out, sh.value


# ------------------------------------------------------------------- PCG
@dataclass
class PCGResult:
    iterations: int
    outer_iterations: int
    rel_residual: float
    solve_ms: float
    status: str


class PCG:
    """IC(0)-PCG (mkl_solver.cpp:150-251 + incomplete_cholesky.cpp:21-29)."""

    def __init__(self, A: CSR, u_ai, u_aj, icc_av, mixed: bool = False):
        self.A = A
        u_ai, u_aj, icc_av = _i32(u_ai), _i32(u_aj), _f64(icc_av)
        h = C.c_void_p()
        call("la_pcg_create", A.h, _ptr(u_ai), _ptr(u_aj), _ptr(icc_av),
             LA_PCG_MIXED if mixed else LA_PCG_FP64, C.byref(h))
        self.h = h

    def solve(self, b, x, rtol=1e-10, maxit=10000, allow_not_converged=False):
        info = PcgInfo()
        ok = (0, 6) if allow_not_converged else (0,)
        if _is_device(b):
            st = call("la_pcg_solve", self.h, _ptr(b), _ptr(x), float(rtol),
                      int(maxit), C.byref(info), _stream(b), ok=ok)
        else:
            b = _f64(b)
            st = call("la_pcg_solve_host", self.h, _ptr(b), _ptr(x),
                      float(rtol), int(maxit), C.byref(info), ok=ok)
        return PCGResult(info.iterations, info.outer_iterations,
                         info.rel_residual, info.solve_ms,
                         _lib.STATUS_NAMES.get(st, str(st)))

    def fused(self):
        """True when each iteration's vector work runs in the two fused
        cooperative kernels (la_pcg_fused)."""
        f = C.c_int()
        call("la_pcg_fused", self.h, C.byref(f))
        return bool(f.value)

    def adjoint(self, g, u, dl_db, dl_dvalues=None, rtol=1e-10, maxit=10000):
        """lambda = A^-T g into dl_db; dL/dA_ij = -lambda_i u_j into dl_dvalues
        (device FP64 tensors)."""
        info = PcgInfo()
        call("la_pcg_adjoint", self.h, _ptr(g), _ptr(u), _ptr(dl_db),
             _ptr(dl_dvalues), float(rtol), int(maxit), C.byref(info), _stream(g))
        return PCGResult(info.iterations, info.outer_iterations, info.rel_residual,
                         info.solve_ms, "LA_OK")

    def __del__(self):
        _release("la_pcg_destroy", self)
