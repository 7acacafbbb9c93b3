"""ctypes bindings for the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  The product path (dcu_b200)
never imports it.

``ref_*`` helpers wrap oracle/_ref/libref_harness.so, the reference's own CPU
helpers compiled from the reference tree; they exist only where that tree was
present at build time.  ``fixture_path`` finds the reference's MatrixMarket
fixtures: the copies the build staged in oracle/_ref/matrices (they travel with
the built files), else the reference tree itself.

The reference tree is found at $DCU_REFERENCE, else at the recipe's default
(oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("DCU_REFERENCE", "/root/reference")
_LIB = None
_REF = None
_EMU = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def reference_present() -> bool:
    return os.path.isdir(os.path.join(REFERENCE, "include", "common"))


def build(reference: str | None = REFERENCE) -> None:
    """Compile liboracle.so (and, when the reference tree exists, the harness
    over its CPU helpers plus the staged copies of its fixtures)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    if reference and os.path.isdir(os.path.join(reference, "include", "common")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "emu", f"REFERENCE={reference}"], check=True)


def fixture_path(name: str) -> str | None:
    """Path of the reference fixture matrices/<name>, or None when neither the
    staged copy nor the reference tree has it."""
    for p in (os.path.join(_HERE, "_ref", "matrices", name), os.path.join(REFERENCE, "matrices", name)):
        if os.path.exists(p):
            return p
    return None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build(None)
        L = C.CDLL(path)
        L.orc_spai_pattern.restype = C.c_longlong
        L.orc_spai_pattern.argtypes = [C.c_int, _i32p, _i32p, C.c_int, C.c_int, _i32p, C.c_void_p, C.c_void_p]
        L.orc_spai_build.restype = C.c_int
        L.orc_spai_build.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, C.c_int, _f64p,
                                     C.c_void_p, C.c_void_p]
        L.orc_csc2csr.restype = None
        L.orc_csc2csr.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.orc_bicgstab.restype = C.c_int
        L.orc_bicgstab.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _f64p, _f64p,
                                   C.c_double, C.c_int, C.c_int, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p]
        L.orc_distribute_columns.restype = None
        L.orc_distribute_columns.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_threads.argtypes = [C.c_int]
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref_harness.so"))


def ref():
    global _REF
    if _REF is None:
        L = C.CDLL(os.path.join(_HERE, "_ref", "libref_harness.so"))
        L.ref_read.restype = C.c_int
        L.ref_read.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_int)),
                               C.POINTER(C.POINTER(C.c_double))]
        L.ref_n1max.restype = C.c_int
        L.ref_n1max.argtypes = [C.c_int, _i32p, _i32p, _f64p]
        L.ref_n1_per_column.restype = None
        L.ref_n1_per_column.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int, _i32p]
        L.ref_n2max.restype = C.c_int
        L.ref_n2max.argtypes = [C.c_int, _i32p, _i32p, _f64p]
        L.ref_csc2csr.restype = None
        L.ref_csc2csr.argtypes = [C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.ref_free.argtypes = [C.c_void_p]
        _REF = L
    return _REF


def emu_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref_emu.so"))


def emu():
    """oracle/_ref/libref_emu.so: the reference's own SPAI kernels on the host
    SIMT emulator and its BiCGSTAB over host stand-ins (ref_emulate.cpp)."""
    global _EMU
    if _EMU is None:
        L = C.CDLL(os.path.join(_HERE, "_ref", "libref_emu.so"))
        L.refemu_spai.restype = C.c_int
        L.refemu_spai.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, C.c_longlong, _i32p]
        L.refemu_bicgstab.restype = C.c_int
        L.refemu_bicgstab.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, C.c_double, C.c_int,
                                      C.POINTER(C.c_double)]
        _EMU = L
    return _EMU


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def refemu_spai(A, tile_budget_bytes: int = 1 << 30):
    """M's values from the reference's own kernels: (mval[nnz], info) with
    info = (n1max, n2max, tiles, single_pass)."""
    mval = np.zeros(max(1, A.nnz), dtype=np.float64)
    info = np.zeros(4, dtype=np.int32)
    rc = emu().refemu_spai(A.n, _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64), mval,
                           int(tile_budget_bytes), info)
    if rc != 0:
        raise RuntimeError(f"refemu_spai failed: {rc}")
    return mval[: A.nnz], tuple(int(v) for v in info)


def refemu_bicgstab(A, mval, b, x0, tol: float, maxiter: int):
    """The reference's cublas2_pbicgstabv2 (absolute ||r|| < tol, counter as
    the reference's): dict(iters, x, res)."""
    x = np.array(x0, dtype=np.float64, copy=True)
    err = C.c_double()
    it = emu().refemu_bicgstab(A.n, _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64),
                               _c(mval, np.float64), _c(b, np.float64), x, float(tol), int(maxiter), C.byref(err))
    return dict(iters=int(it), x=x, res=err.value)


def set_threads(t: int) -> None:
    lib().orc_set_threads(int(t))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def pattern(A, col_start: int = 0, col_end: int | None = None):
    """(icount[k], iptr, ilist): sorted unions I_k for k in [col_start, col_end)."""
    col_end = A.n if col_end is None else col_end
    ptr, idx = _c(A.ptr, np.int32), _c(A.idx, np.int32)
    cnt = np.zeros(col_end - col_start, dtype=np.int32)
    lib().orc_spai_pattern(A.n, ptr, idx, col_start, col_end, cnt, None, None)
    iptr = np.zeros(len(cnt) + 1, dtype=np.int64)
    np.cumsum(cnt, out=iptr[1:])
    ilist = np.zeros(max(1, int(iptr[-1])), dtype=np.int32)
    lib().orc_spai_pattern(A.n, ptr, idx, col_start, col_end, cnt, iptr.ctypes.data, ilist.ctypes.data)
    return cnt, iptr, ilist[: int(iptr[-1])]


def spai(A, method: str = "mgs", col_start: int = 0, col_end: int | None = None):
    """SPAI values on A's pattern: (mval[nnz], colres[ncols], E[ncols], n_singular).

    method "mgs" follows the reference's modified Gram-Schmidt + Sol order;
    "householder" is the FP64 accuracy oracle.  Columns outside the range stay 0.
    """
    col_end = A.n if col_end is None else col_end
    ptr, idx, val = _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64)
    mval = np.zeros(A.nnz, dtype=np.float64)
    colres = np.zeros(col_end - col_start, dtype=np.float64)
    E = np.zeros(col_end - col_start, dtype=np.int32)
    sing = lib().orc_spai_build(A.n, ptr, idx, val, col_start, col_end, 0 if method == "mgs" else 1,
                                mval, colres.ctypes.data, E.ctypes.data)
    return mval, colres, E, int(sing)


def csc2csr(n, ptr, idx, val):
    ptr, idx, val = _c(ptr, np.int32), _c(idx, np.int32), _c(val, np.float64)
    rp = np.zeros(n + 1, dtype=np.int32)
    ri = np.zeros(max(1, len(idx)), dtype=np.int32)
    rv = np.zeros(max(1, len(idx)), dtype=np.float64)
    lib().orc_csc2csr(n, ptr, idx, val, rp, ri, rv)
    return rp, ri[: len(idx)], rv[: len(idx)]


def bicgstab(A, mval, b, x0=None, tol=1e-8, tol_mode="rel", maxiter=1000, history=False):
    """Reference-order BiCGSTAB with M on A's pattern.

    Returns dict(iters, x, res (recurrence ||r||), true_res (||b - A x||),
    status, hist)."""
    n = A.n
    Arp, Aci, Arv = csc2csr(n, A.ptr, A.idx, A.val)
    Mrp, Mci, Mrv = csc2csr(n, A.ptr, A.idx, mval)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    b = _c(b, np.float64)
    fr, tr, st = C.c_double(), C.c_double(), C.c_int()
    hist = np.zeros(max(1, maxiter), dtype=np.float64) if history else None
    it = lib().orc_bicgstab(n, Arp, Aci, Arv, Mrp, Mci, Mrv, b, x, tol, 1 if tol_mode == "rel" else 0,
                            maxiter, C.byref(fr), C.byref(tr), C.byref(st),
                            hist.ctypes.data if history else None)
    out = dict(iters=int(it), x=x, res=fr.value, true_res=tr.value, status=int(st.value))
    if history:
        out["hist"] = hist[: max(0, it)]
    return out


def distribute_columns(ptr, col_start, col_end, units, use_nnz):
    s = np.zeros(units, dtype=np.int32)
    e = np.zeros(units, dtype=np.int32)
    lib().orc_distribute_columns(_c(ptr, np.int32), col_start, col_end, units, 1 if use_nnz else 0, s, e)
    return s, e


def _take_csc(n, nnz, p, i, v, free):
    from dcu_b200.workloads import CSC

    if n == 0 or not p:
        return CSC(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    ptr = np.ctypeslib.as_array(p, shape=(n + 1,)).copy()
    idx = np.ctypeslib.as_array(i, shape=(max(nnz, 1),))[:nnz].copy()
    val = np.ctypeslib.as_array(v, shape=(max(nnz, 1),))[:nnz].copy()
    for q in (p, i, v):
        free(C.cast(q, C.c_void_p))
    return CSC(n, ptr, idx, val)


def ref_mtx_read(path: str):
    n, nnz = C.c_int(), C.c_int()
    p, i, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    ref().ref_read(path.encode(), C.byref(n), C.byref(nnz), C.byref(p), C.byref(i), C.byref(v))
    return _take_csc(n.value, nnz.value, p, i, v, ref().ref_free)


def ref_n1max(A) -> int:
    return int(ref().ref_n1max(A.n, _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64)))


def ref_n1_per_column(A, col_start: int = 0, col_end: int | None = None):
    """|I_k| of each column from the reference's computeN1MAX on a one-column M."""
    col_end = A.n if col_end is None else col_end
    out = np.zeros(max(1, col_end - col_start), dtype=np.int32)
    ref().ref_n1_per_column(A.n, _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64),
                            col_start, col_end, out)
    return out[: col_end - col_start]


def ref_n2max(A) -> int:
    return int(ref().ref_n2max(A.n, _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64)))


def ref_csc2csr(A):
    rp = np.zeros(A.n + 1, dtype=np.int32)
    ri = np.zeros(max(1, A.nnz), dtype=np.int32)
    rv = np.zeros(max(1, A.nnz), dtype=np.float64)
    ref().ref_csc2csr(A.n, _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64), rp, ri, rv)
    return rp, ri[: A.nnz], rv[: A.nnz]
