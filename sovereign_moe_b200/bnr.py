"""Batched node relaxation on the B200: drop-in for ``sovopt.mip.bnr``.

``BNREngine(prob, scaling, config)`` and ``solve_batch(col_lb, col_ub,
warm=None) -> BatchResult`` keep the reference's interface
(``src/sovopt/mip/bnr.py:90-301``).  K node LPs share one pdlp-scaled
problem and differ only in their column bounds.  They advance together by
``config.iters`` PDHG iterations with a step size per node, and each gets the
safe dual bound of its dual iterate (``src/sovopt/mip/safebound.py:194-235``).
The work runs in ``libpdlp_b200.so`` (``csrc/bnr.cu``): sparse products over
(rows, K) node-fastest blocks, which read the matrix once for all K nodes;
fused element-wise steps; per-node sums; and the iterations of a call
replayed from a CUDA graph.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

__all__ = ["BNRConfig", "BNREngine", "BatchResult"]


@dataclass
class BNRConfig:
    """``BNRConfig`` (bnr.py:90-108)."""
    batch: int = 128
    iters: int = 60
    warm_start: bool = True
    eps: float = 1e-9
    device: str = "auto"
    step_growth: float = 0.3
    step_damp: float = 0.6


@dataclass
class BatchResult:
    """``BatchResult`` (bnr.py:111-122), plus the dual iterate ``y`` (m, K)
    that the reference's tree reads from ``engine.Y``."""
    bounds: np.ndarray
    x: np.ndarray
    iterations: int = 0
    infeasible: np.ndarray | None = None
    y: np.ndarray | None = None


class _HostView:
    """``engine.bk`` for callers written against the reference engine, which
    read ``engine.bk.to_host(engine.Y[:, :K])`` (mip/tree.py:1025): the
    iterates this engine returns are already host arrays."""

    @staticmethod
    def to_host(a):
        return np.asarray(a)


class BNREngine:
    """Holds the shared scaled problem on the device and advances node batches."""

    def __init__(self, prob, scaling, config: BNRConfig | None = None):
        self.cfg = config or BNRConfig()
        if self.cfg.device == "cpu":
            raise ValueError("this BNR engine runs on the GPU only: use device='gpu' or 'auto'")
        self.lib = _lib.load()
        self.prob = prob
        self.m, self.n = int(prob.A.m), int(prob.A.n)
        A = prob.A
        self._keep = dict(
            rp=np.ascontiguousarray(A.rp, np.int64), ri=np.ascontiguousarray(A.ri, np.int32),
            rx=np.ascontiguousarray(A.rx, np.float64), cp=np.ascontiguousarray(A.cp, np.int64),
            ci=np.ascontiguousarray(A.ci, np.int32), cx=np.ascontiguousarray(A.cx, np.float64),
            c=np.ascontiguousarray(prob.c, np.float64),
            row_lb=np.ascontiguousarray(prob.row_lb, np.float64),
            row_ub=np.ascontiguousarray(prob.row_ub, np.float64))
        d = _lib.ProblemDesc()
        d.m, d.n, d.nnz = self.m, self.n, int(self._keep["ci"].shape[0])
        for k, a in self._keep.items():
            setattr(d, k, a.ctypes.data if a.size else None)
        d.rp, d.cp = self._keep["rp"].ctypes.data, self._keep["cp"].ctypes.data
        d.obj_offset = float(prob.obj_offset)
        d.sense = 1
        d.memory = _lib.PDLP_MEM_HOST
        self.obj_scale = float(getattr(scaling, "obj", 1.0) or 1.0)
        h = ctypes.c_void_p()
        code = self.lib.pdlp_bnr_create(ctypes.byref(d), self.obj_scale, int(self.cfg.batch),
                                        None, ctypes.byref(h))
        if code == _lib.PDLP_ERR_CUDA:
            raise RuntimeError(f"GPU backend unavailable ({self.lib.pdlp_last_error().decode()})")
        _lib.check(code)
        self.h = h
        self.bk = _HostView()
        self._cap = max(1, int(self.cfg.batch))
        self.total_iterations = 0
        self.total_batches = 0
        self.total_nodes = 0
        self._last_y = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.pdlp_bnr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def Y(self):
        """The dual iterates (m, K) of the last batch (the reference keeps them
        on its engine; its tree caches them as warm starts)."""
        return self._last_y

    @property
    def eta(self):
        """Step sizes of every node slot (bnr.py:168-171)."""
        return self.step_sizes(self._cap)[0]

    @property
    def omega(self):
        return self.step_sizes(self._cap)[1]

    def step_sizes(self, K):
        eta = np.empty(K)
        omega = np.empty(K)
        _lib.check(self.lib.pdlp_bnr_step_sizes(self.h, int(K), eta.ctypes.data,
                                                omega.ctypes.data))
        return eta, omega

    def solve_batch(self, col_lb, col_ub, warm=None) -> BatchResult:
        """Advance ``K`` nodes and return valid lower bounds for each
        (bnr.py:176-301).  ``col_lb`` / ``col_ub`` are ``(n, K)`` arrays of
        per-node bounds in the scaled space; ``warm`` is an optional ``(X, Y)``
        pair of ``(n, K)`` and ``(m, K)`` arrays."""
        L = np.ascontiguousarray(col_lb, dtype=np.float64)
        U = np.ascontiguousarray(col_ub, dtype=np.float64)
        if L.ndim != 2 or L.shape != U.shape or L.shape[0] != self.n:
            raise ValueError("col_lb and col_ub must both be (n, K)")
        K = int(L.shape[1])
        wx = wy = None
        if warm is not None:
            wx = np.ascontiguousarray(warm[0], dtype=np.float64)
            wy = np.ascontiguousarray(warm[1], dtype=np.float64)
            if wx.shape != (self.n, K) or wy.shape != (self.m, K):
                raise ValueError("warm must be ((n, K), (m, K)) arrays")
        bounds = np.empty(K)
        x = np.empty((self.n, K))
        y = np.empty((self.m, K))
        inf = np.empty(K, dtype=np.uint8)
        _lib.check(self.lib.pdlp_bnr_solve_batch(
            self.h, K, L.ctypes.data, U.ctypes.data,
            wx.ctypes.data if wx is not None else None,
            wy.ctypes.data if wy is not None else None,
            int(self.cfg.iters), float(self.cfg.step_growth), float(self.cfg.step_damp),
            bounds.ctypes.data, x.ctypes.data, y.ctypes.data, inf.ctypes.data,
            _lib.PDLP_MEM_HOST))
        self._last_y = y
        if K > self._cap:
            self._cap = max(K, 2 * self._cap)
        self.total_iterations += self.cfg.iters
        self.total_batches += 1
        self.total_nodes += K
        return BatchResult(bounds=bounds, x=x, iterations=self.cfg.iters,
                           infeasible=inf.astype(bool), y=y)

    def stats(self) -> dict:
        """bnr.py:305-312."""
        return {"device": "gpu", "batches": self.total_batches,
                "nodes_bounded": self.total_nodes, "pdhg_iterations": self.total_iterations,
                "avg_batch": self.total_nodes / max(self.total_batches, 1)}

    def __repr__(self):
        return (f"BNREngine({self.m}x{self.n} on gpu, batch={self.cfg.batch}, "
                f"iters={self.cfg.iters})")
