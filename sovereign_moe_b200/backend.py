"""Kernel-level API mirroring the reference ``Backend`` on torch CUDA tensors.

The reference writes its first-order method against ``sovopt.core.backend.
Backend`` (``src/sovopt/core/backend.py:317-493``).  This class keeps that
surface -- ``spmv``, ``spmm``, ``primal_step``, ``dual_step``,
``pdhg_primal``, ``pdhg_dual``, ``pdhg_accum``, ``dot``, ``nrm2``,
``nrm_inf`` plus the transfer helpers -- for ``device="gpu"`` only, with torch
providing device memory and the current CUDA stream.  Each method calls the
matching entry point of ``libpdlp_b200.so``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

__all__ = ["Backend", "SpmvPlan", "get_backend", "gpu_selftest"]


def _torch():
    import torch
    return torch


class SpmvPlan:
    """A planned ``y = A x`` on one sparsity pattern (``pdlp_spmv_plan_*``).

    The reference multiplies by the same ``A`` and ``A^T`` at every PDHG
    iteration (``backend.py:373-384``); the plan analyses the pattern once --
    tiles of rows, each with the column window and halo its ``x`` gathers come
    from -- and each ``run`` is one persistent kernel that streams the matrix
    into shared memory.  The plan copies ``rp`` and ``ri`` (int64 / int32
    device tensors); the values are passed to each run and may change.
    """

    def __init__(self, lib, rp, ri, m, n, stream):
        self.lib = lib
        self.m, self.n = int(m), int(n)
        h = ctypes.c_void_p()
        _lib.check(lib.pdlp_spmv_plan_create(self.m, self.n, rp.data_ptr(), ri.data_ptr(),
                                             stream, ctypes.byref(h)))
        self._h = h

    def run(self, rx, x, out, stream):
        torch = _torch()
        fn = (self.lib.pdlp_spmv_plan_run_f32 if rx.dtype == torch.float32
              else self.lib.pdlp_spmv_plan_run_f64)
        _lib.check(fn(self._h, rx.data_ptr(), x.data_ptr(), out.data_ptr(), stream))
        return out

    def info(self) -> dict:
        i = _lib.SpmvPlanInfo()
        _lib.check(self.lib.pdlp_spmv_plan_get_info(self._h, ctypes.byref(i)))
        return {f: getattr(i, f) for f, _ in i._fields_}

    def status(self, stream) -> int:
        return int(self.lib.pdlp_spmv_plan_status(self._h, stream))

    def close(self):
        if self._h:
            self.lib.pdlp_spmv_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Backend:
    """Array namespace plus sparse kernels on the GPU (``backend.py:317-327``)."""

    def __init__(self, device: str = "gpu", dtype=np.float64, autotune: bool = False):
        if device not in ("cpu", "gpu"):
            raise ValueError("device must be 'cpu' or 'gpu'")
        if device == "cpu":
            raise ValueError("this backend runs on the GPU only")
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("GPU backend unavailable (no CUDA device)")
        self.lib = _lib.load()
        self.device = "gpu"
        self.dtype = np.dtype(dtype)
        self._tdtype = torch.float32 if self.dtype == np.float32 else torch.float64
        # autotune: the first spmv on a matrix times the kernel's variants on
        # it (pdlp_spmv_tune_*) and later calls use the fastest.  The choice is
        # keyed by the matrix arrays' device addresses; a stale key costs only
        # speed, since every variant computes the same product.
        self.autotune = bool(autotune)
        self._spmv_variant = {}

    # -- transfer ------------------------------------------------------------ #

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)

    def to_device(self, a, dtype=None):
        torch = _torch()
        dt = self._tdtype if dtype is None else {
            np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
            np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}[np.dtype(dtype)]
        return torch.as_tensor(np.ascontiguousarray(a), device="cuda").to(dt).contiguous()

    def to_host(self, a):
        return a.detach().cpu().numpy()

    def index(self, a):
        return self.to_device(a, dtype=np.int32)

    def pointer(self, a):
        return self.to_device(a, dtype=np.int64)

    def sync(self):
        _torch().cuda.current_stream().synchronize()

    def zeros(self, shape, dtype=None):
        return _torch().zeros(shape, dtype=self._tdtype if dtype is None else dtype, device="cuda")

    def empty(self, shape, dtype=None):
        return _torch().empty(shape, dtype=self._tdtype if dtype is None else dtype, device="cuda")

    # -- sparse products ------------------------------------------------------ #

    def spmv(self, rp, ri, rx, x, out, m):
        """``out = A x`` with ``A`` in CSR (``backend.py:373-384``)."""
        torch = _torch()
        f32 = rx.dtype == torch.float32
        if not self.autotune:
            fn = self.lib.pdlp_spmv_f32 if f32 else self.lib.pdlp_spmv_f64
            _lib.check(fn(int(m), rp.data_ptr(), ri.data_ptr(), rx.data_ptr(), x.data_ptr(),
                          out.data_ptr(), self._stream()))
            return out
        key = (rp.data_ptr(), ri.data_ptr(), rx.data_ptr(), int(m), f32)
        variant = self._spmv_variant.get(key)
        if variant is None:
            best = ctypes.c_int32(0)
            tune = self.lib.pdlp_spmv_tune_f32 if f32 else self.lib.pdlp_spmv_tune_f64
            _lib.check(tune(int(m), rp.data_ptr(), ri.data_ptr(), rx.data_ptr(), x.data_ptr(),
                            out.data_ptr(), self._stream(), 10, ctypes.byref(best), None))
            self._spmv_variant[key] = best.value
            return out
        fn = self.lib.pdlp_spmv_ex_f32 if f32 else self.lib.pdlp_spmv_ex_f64
        _lib.check(fn(int(variant), int(m), rp.data_ptr(), ri.data_ptr(), rx.data_ptr(),
                      x.data_ptr(), out.data_ptr(), self._stream()))
        return out

    def spmv_plan(self, rp, ri, m, n) -> SpmvPlan:
        """A plan for repeated ``A x`` on this pattern (synchronises the stream)."""
        return SpmvPlan(self.lib, rp, ri, m, n, self._stream())

    def spmv_planned(self, plan: SpmvPlan, rx, x, out):
        """``out = A x`` through a plan made by :meth:`spmv_plan`."""
        return plan.run(rx, x, out, self._stream())

    def spmm(self, rp, ri, rx, X, out, m, k_batch):
        """``out = A X``, ``X`` dense ``(n, k)`` row-major (``backend.py:386-400``)."""
        _lib.check(self.lib.pdlp_spmm_f64(int(m), int(k_batch), rp.data_ptr(), ri.data_ptr(),
                                          rx.data_ptr(), X.data_ptr(), out.data_ptr(),
                                          self._stream()))
        return out

    # -- fused steps -------------------------------------------------------- #

    def primal_step(self, xnew, x, c, aty, lo, hi, tau, n):
        _lib.check(self.lib.pdlp_primal_step(int(n), xnew.data_ptr(), x.data_ptr(), c.data_ptr(),
                                             aty.data_ptr(), lo.data_ptr(), hi.data_ptr(),
                                             float(tau), self._stream()))
        return xnew

    def dual_step(self, ynew, y, ax, rl, ru, sigma, m):
        _lib.check(self.lib.pdlp_dual_step(int(m), ynew.data_ptr(), y.data_ptr(), ax.data_ptr(),
                                           rl.data_ptr(), ru.data_ptr(), float(sigma),
                                           self._stream()))
        return ynew

    def pdhg_primal(self, x, dx, c, aty, lo, hi, tau, n):
        _lib.check(self.lib.pdlp_pdhg_primal(int(n), x.data_ptr(), dx.data_ptr(), c.data_ptr(),
                                             aty.data_ptr(), lo.data_ptr(), hi.data_ptr(),
                                             float(tau), self._stream()))

    def pdhg_dual(self, y, dy, ax, adx, rl, ru, sigma, m):
        _lib.check(self.lib.pdlp_pdhg_dual(int(m), y.data_ptr(), dy.data_ptr(), ax.data_ptr(),
                                           adx.data_ptr(), rl.data_ptr(), ru.data_ptr(),
                                           float(sigma), self._stream()))

    def pdhg_accum(self, acc, inc, run_sum, v, eta, n):
        _lib.check(self.lib.pdlp_pdhg_accum(int(n), acc.data_ptr(), inc.data_ptr(),
                                            run_sum.data_ptr(), v.data_ptr(), float(eta),
                                            self._stream()))

    # -- reductions --------------------------------------------------------- #

    def dot(self, a, b) -> float:
        out = ctypes.c_double()
        _lib.check(self.lib.pdlp_dot(int(a.numel()), a.data_ptr(), b.data_ptr(),
                                     ctypes.byref(out), self._stream()))
        return out.value

    def nrm2(self, a) -> float:
        out = ctypes.c_double()
        _lib.check(self.lib.pdlp_nrm2(int(a.numel()), a.data_ptr(), ctypes.byref(out),
                                      self._stream()))
        return out.value

    def nrm_inf(self, a) -> float:
        out = ctypes.c_double()
        _lib.check(self.lib.pdlp_nrm_inf(int(a.numel()), a.data_ptr() if a.numel() else 0,
                                         ctypes.byref(out), self._stream()))
        return out.value

    def __repr__(self):
        return f"Backend(gpu, {self.dtype.name})"


_SELFTEST = None


def gpu_selftest():
    """Build the kernels and check one known answer (``backend.py:499-535``):
    ``[[1, 0, 2], [0, 3, 0]] @ [1, 2, 3] = [7, 6]``.  Cached."""
    global _SELFTEST
    if _SELFTEST is not None:
        return _SELFTEST
    try:
        bk = Backend("gpu")
        rp = bk.pointer(np.array([0, 2, 3], dtype=np.int64))
        ri = bk.index(np.array([0, 2, 1], dtype=np.int32))
        rx = bk.to_device(np.array([1.0, 2.0, 3.0]))
        x = bk.to_device(np.array([1.0, 2.0, 3.0]))
        y = bk.zeros(2)
        bk.spmv(rp, ri, rx, x, y, 2)
        bk.sync()
        got = bk.to_host(y)
        _SELFTEST = (True, None) if np.array_equal(got, [7.0, 6.0]) else \
            (False, f"spmv returned {got.tolist()}, expected [7.0, 6.0]")
    except Exception as exc:      # pragma: no cover - environment dependent
        _SELFTEST = (False, f"{type(exc).__name__}: {exc}")
    return _SELFTEST


def get_backend(device: str = "auto", dtype=np.float64) -> Backend:
    """``'auto'`` and ``'gpu'`` both need a usable GPU (no CPU fallback)."""
    if device == "cpu":
        raise ValueError("this backend runs on the GPU only")
    ok, err = gpu_selftest()
    if not ok:
        raise RuntimeError(f"GPU backend unavailable ({err})")
    return Backend("gpu", dtype)
