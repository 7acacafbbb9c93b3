"""Python face of the library for tests and the benchmark.

Host arrays are numpy; device arrays are torch CUDA tensors (torch is only
the allocator and stream here, every computation runs in libdcu_spai.so).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .workloads import CSC


class DcuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"status {status}: {msg}")
        self.status = status


def _p(a) -> int:
    """Raw pointer of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    assert a.is_contiguous()
    return a.data_ptr()


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class Context:
    """A dcu_spai_ctx on one CUDA device (replaces initMultiDCU/cleanupMultiDCU)."""

    def __init__(self, device: int = 0, units: int = 0):
        self._L = N.lib()
        h = C.c_void_p()
        rc = self._L.dcu_spai_create(C.byref(h), device, units)
        if rc != N.OK:
            raise DcuError(rc, "dcu_spai_create failed")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self._L.dcu_spai_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- helpers
    def _check(self, rc):
        if rc != N.OK:
            raise DcuError(rc, self._L.dcu_spai_last_error(self.h).decode())

    @property
    def units(self) -> int:
        return int(self._L.dcu_spai_units(self.h))

    @property
    def launches(self) -> int:
        return int(self._L.dcu_spai_launch_count(self.h))

    def set_stream(self, stream_ptr: int | None):
        self._check(self._L.dcu_spai_set_stream(self.h, stream_ptr))

    # ------------------------------------------------------------ host entry
    def build_h(self, A: CSC, **opt):
        """SPAI values on A's pattern (host arrays) -> (mval, colres, BuildInfo)."""
        o = N.default_options(**opt)
        ptr, idx, val = _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64)
        mval = np.zeros(A.nnz, dtype=np.float64)
        ce = o.col_end if o.col_end > 0 else A.n
        colres = np.zeros(max(1, ce - o.col_start), dtype=np.float64)
        info = N.BuildInfo()
        self._check(self._L.dcu_spai_build_h(self.h, A.n, A.nnz, _p(ptr), _p(idx), _p(val), C.byref(o), _p(mval),
                                             _p(colres), C.byref(info)))
        return mval, colres[: ce - o.col_start], info

    def bicgstab_h(self, A: CSC, mval, b, x0=None, **opt):
        o = N.default_options(**opt)
        ptr, idx, val = _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64)
        m = _c(mval, np.float64)
        b = _c(b, np.float64)
        x = np.zeros(A.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        info = N.SolveInfo()
        self._check(self._L.dcu_bicgstab_h(self.h, A.n, A.nnz, _p(ptr), _p(idx), _p(val), _p(m), _p(b), _p(x),
                                           C.byref(o), C.byref(info)))
        return x, info

    def solve_h(self, A: CSC, b, x0=None, want_m=False, **opt):
        o = N.default_options(**opt)
        ptr, idx, val = _c(A.ptr, np.int32), _c(A.idx, np.int32), _c(A.val, np.float64)
        b = _c(b, np.float64)
        x = np.zeros(A.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        mval = np.zeros(A.nnz, dtype=np.float64) if want_m else None
        bi, si = N.BuildInfo(), N.SolveInfo()
        self._check(self._L.dcu_spai_solve_h(self.h, A.n, A.nnz, _p(ptr), _p(idx), _p(val), _p(b), _p(x), C.byref(o),
                                             _p(mval), C.byref(bi), C.byref(si)))
        return x, mval, bi, si

    def solve_h_into(self, n, nnz, ptr, idx, val, b, x, mval=None, **opt):
        """dcu_spai_solve_h on caller-owned host arrays used as they are
        (pinned memory stays pinned); x holds x0 on entry, the solution on exit."""
        for a, dt in ((ptr, np.int32), (idx, np.int32), (val, np.float64), (b, np.float64), (x, np.float64)):
            assert a.dtype == dt and a.flags["C_CONTIGUOUS"]
        o = N.default_options(**opt)
        bi, si = N.BuildInfo(), N.SolveInfo()
        self._check(self._L.dcu_spai_solve_h(self.h, n, nnz, _p(ptr), _p(idx), _p(val), _p(b), _p(x), C.byref(o),
                                             _p(mval), C.byref(bi), C.byref(si)))
        return bi, si

    # ---------------------------------------------------------- device entry
    def pattern_d(self, n, ptr_d, idx_d, col_start=0, col_end=None):
        """(icount, iptr, ilist) as torch tensors on the device."""
        import torch

        col_end = n if col_end is None else col_end
        ncols = col_end - col_start
        dev = ptr_d.device
        icount = torch.zeros(max(1, ncols), dtype=torch.int32, device=dev)
        iptr = torch.zeros(ncols + 1, dtype=torch.int64, device=dev)
        total = C.c_longlong()
        self._check(self._L.dcu_spai_pattern_d(self.h, n, _p(ptr_d), _p(idx_d), col_start, col_end, _p(icount),
                                               _p(iptr), None, 0, C.byref(total)))
        ilist = torch.zeros(max(1, total.value), dtype=torch.int32, device=dev)
        self._check(self._L.dcu_spai_pattern_d(self.h, n, _p(ptr_d), _p(idx_d), col_start, col_end, _p(icount),
                                               _p(iptr), _p(ilist), ilist.numel(), C.byref(total)))
        return icount[:ncols], iptr, ilist[: total.value]

    def build_d(self, n, nnz, ptr_d, idx_d, val_d, mval_d, colres_d=None, **opt):
        o = N.default_options(**opt)
        info = N.BuildInfo()
        self._check(self._L.dcu_spai_build_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(val_d), C.byref(o),
                                             _p(mval_d), _p(colres_d), C.byref(info)))
        return info

    def profile_iteration(self, reps: int = 20):
        ms = (C.c_float * 16)()
        cnt = C.c_int(0)
        self._check(self._L.dcu_profile_iteration_kernels(self.h, reps, ms, 16, C.byref(cnt)))
        return [float(ms[i]) for i in range(cnt.value)]

    def sell_plan_stats(self, wide: bool = False):
        """(slots, uniform_slots) of the last SELL layout built on this context; with wide=True also the
        number of full slices made wider than 16 slots by at most 4 long rows (summed by the warp-cooperative
        pre-pass)."""
        s, u, w = C.c_longlong(), C.c_longlong(), C.c_longlong()
        self._check(self._L.dcu_sell_plan_stats(self.h, C.byref(s), C.byref(u), C.byref(w)))
        return (s.value, u.value, w.value) if wide else (s.value, u.value)

    def set_wide_prepass(self, enabled: bool):
        """Wide-slice pre-pass of later solves on (default) or off (dcu_set_wide_prepass)."""
        self._check(self._L.dcu_set_wide_prepass(self.h, 1 if enabled else 0))

    def set_exact_a32(self, enabled: bool):
        """A read from its FP32 copy when every value is exact in FP32 (default), or always FP64
        (dcu_set_exact_a32); the iterates are bit-identical either way."""
        self._check(self._L.dcu_set_exact_a32(self.h, 1 if enabled else 0))

    def autotune_d(self, n, nnz, ptr_d, idx_d, val_d, b_d, reps: int = 10, **opt) -> "N.Tuning":
        """Time the launch configurations of opt's precision form on this matrix and keep the fastest
        for later builds and solves of that form on this context (dcu_autotune_d)."""
        o = N.default_options(**opt)
        t = N.Tuning()
        self._check(self._L.dcu_autotune_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(val_d), _p(b_d), C.byref(o),
                                           reps, C.byref(t)))
        return t

    def set_tuning(self, precision: int, tuning: "N.Tuning | None" = None, **fields):
        """Pin a launch configuration for one precision form (None and no fields: back to the defaults)."""
        if tuning is None and not fields:
            self._check(self._L.dcu_set_tuning(self.h, precision, None))
            return
        t = N.Tuning()
        if tuning is not None:
            C.pointer(t)[0] = tuning
        else:
            self._L.dcu_tuning_default(C.byref(t))
        for k, v in fields.items():
            if k not in N.Tuning.CONFIG:
                raise KeyError(k)
            setattr(t, k, v)
        self._check(self._L.dcu_set_tuning(self.h, precision, C.byref(t)))

    def get_tuning(self, precision: int) -> "N.Tuning":
        t = N.Tuning()
        self._check(self._L.dcu_get_tuning(self.h, precision, C.byref(t)))
        return t

    def csc_to_csr_d(self, n, nnz, ptr_d, idx_d, val_d, rptr_d, ridx_d, rval_d):
        self._check(self._L.dcu_csc_to_csr_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(val_d), _p(rptr_d),
                                             _p(ridx_d), _p(rval_d)))

    def bicgstab_d(self, n, nnz, ptr_d, idx_d, val_d, mval_d, b_d, x_d, **opt):
        o = N.default_options(**opt)
        info = N.SolveInfo()
        self._check(self._L.dcu_bicgstab_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(val_d), _p(mval_d), _p(b_d),
                                           _p(x_d), C.byref(o), C.byref(info)))
        return info

    def bicgstab_transpose_d(self, n, nnz, ptr_d, idx_d, val_d, mval_d, b_d, x_d, **opt):
        """A^T x = b with preconditioner M^T (the adjoint solve)."""
        o = N.default_options(**opt)
        info = N.SolveInfo()
        self._check(self._L.dcu_bicgstab_transpose_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(val_d), _p(mval_d),
                                                     _p(b_d), _p(x_d), C.byref(o), C.byref(info)))
        self.last_adjoint = info
        return info

    def sampled_outer_d(self, n, nnz, ptr_d, idx_d, u_d, v_d, alpha, out_d):
        self._check(self._L.dcu_sampled_outer_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(u_d), _p(v_d),
                                                float(alpha), _p(out_d)))

    def batch_solve_d(self, sys_off_d, n, nnz, ptr_d, idx_d, val_d, B_d, X_d, mval_d=None, **opt):
        """Independent diagonal-block systems x nrhs (B_d, X_d: n x nrhs).
        Returns (iters[nsys, nrhs], status[nsys, nrhs], BuildInfo, SolveInfo)."""
        o = N.default_options(**opt)
        nsys = sys_off_d.numel() - 1
        nrhs = B_d.shape[1]
        iters = np.zeros(nsys * nrhs, dtype=np.int32)
        status = np.zeros(nsys * nrhs, dtype=np.int32)
        bi, si = N.BuildInfo(), N.SolveInfo()
        self._check(self._L.dcu_batch_solve_d(self.h, nsys, _p(sys_off_d), n, nnz, _p(ptr_d), _p(idx_d),
                                              _p(val_d), nrhs, _p(B_d), _p(X_d), C.byref(o), _p(mval_d),
                                              _p(iters), _p(status), C.byref(bi), C.byref(si)))
        return iters.reshape(nsys, nrhs), status.reshape(nsys, nrhs), bi, si

    def solve_d(self, n, nnz, ptr_d, idx_d, val_d, b_d, x_d, mval_d=None, **opt):
        o = N.default_options(**opt)
        bi, si = N.BuildInfo(), N.SolveInfo()
        self._check(self._L.dcu_spai_solve_d(self.h, n, nnz, _p(ptr_d), _p(idx_d), _p(val_d), _p(b_d), _p(x_d),
                                             C.byref(o), _p(mval_d), C.byref(bi), C.byref(si)))
        self.last_solve = (bi, si)
        return bi, si


def distribute_columns(ptr, col_start, col_end, units, schedule):
    """distributeColumns through the C ABI (host computation)."""
    ptr = _c(ptr, np.int32)
    s = np.zeros(units, dtype=np.int32)
    e = np.zeros(units, dtype=np.int32)
    rc = N.lib().dcu_spai_distribute_columns(_p(ptr), col_start, col_end, units, schedule, _p(s), _p(e))
    if rc != N.OK:
        raise DcuError(rc, "dcu_spai_distribute_columns")
    return s, e


def mtx_read(path: str) -> CSC:
    """MatrixMarket -> CSC with the reference reader's semantics (C ABI)."""
    L = N.lib()
    n, nnz = C.c_int(), C.c_int()
    p, i, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    rc = L.dcu_mtx_read(path.encode(), C.byref(n), C.byref(nnz), C.byref(p), C.byref(i), C.byref(v))
    if rc != 0:
        raise IOError(f"dcu_mtx_read({path}) failed: {rc}")
    if n.value == 0 or not p:
        return CSC(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    nz = nnz.value
    out = CSC(n.value, np.ctypeslib.as_array(p, shape=(n.value + 1,)).copy(),
              np.ctypeslib.as_array(i, shape=(max(nz, 1),))[:nz].copy(),
              np.ctypeslib.as_array(v, shape=(max(nz, 1),))[:nz].copy())
    for q in (p, i, v):
        L.dcu_mtx_free(C.cast(q, C.c_void_p))
    return out
