"""CPU oracle of the batched node relaxation (BNR): test infrastructure only.

A restatement, in this repository's own code, of the reference's
``BNREngine.solve_batch`` (``src/sovopt/mip/bnr.py:176-301``) and of
``safe_dual_bound_batch`` (``src/sovopt/mip/safebound.py:194-235``) on the
reference's CPU backend, where the array namespace is NumPy and ``spmm`` is
the row-wise CSR kernel of ``src/sovopt/core/sparse.py:72-84``.  The oracle
makes the same NumPy calls in the same order, so it reproduces the
reference's CPU results bit for bit.  ``tests/golden/bnr/*.npz``, made by
``tests/golden/bnr/make_golden_bnr.py`` from the reference itself, pin it.

``sum_order="tree"`` replaces the per-node sums over rows (the step-size
test's three inner products and the two halves of the safe bound) by the
device engine's fixed order, and leaves every other operation as it is:
blocks of 64 rows, each the sum of 8 phases (rows ``b*64 + y + 8 j``, ``j``
ascending) added in phase order; then 32 lanes, lane ``l`` adding blocks
``l, l + 32, ...`` in order; then the lanes in order.  With it the oracle predicts the
device engine bit for bit; the default ``"sequential"`` is the reference's
NumPy order.

Only ``tests/`` may use this module, to check the device engine
(``sovereign_moe_b200.bnr``) against it.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from . import pdlp_oracle as po

INF = 1.0e30                 # core/tolerances.py:16
QUOTIENT_MAX = 2.0 ** 1000   # core/tolerances.py:23


def sum_rows(P):
    """``P.sum(axis=0)`` for a C-ordered (rows, K) block: NumPy adds the rows
    one after another."""
    return P.sum(axis=0)


def sum_rows_tree(P, block=64, phases=8):
    """The device engine's per-node sum over rows (``bnr_block_sums`` and
    ``warp_blocks_sum`` in csrc/bnr.cu): per block of 64 rows, phase ``y``
    adds rows ``y, y + 8, ...`` from 0.0 and the phases are added in order;
    lane ``l`` of 32 adds blocks ``l, l + 32, ...`` in order from 0.0; the
    lane sums are added in lane order."""
    rows, K = P.shape
    nb = -(-rows // block)
    Q = np.zeros((nb * block, K))
    Q[:rows] = P
    Q = Q.reshape(nb, block // phases, phases, K)     # (block, j, phase y, node)
    s = np.zeros((nb, phases, K))
    for j in range(block // phases):
        s = s + Q[:, j]
    a = s[:, 0]
    for y in range(1, phases):
        a = a + s[:, y]
    lanes = np.zeros((32, K))
    for b in range(nb):
        lanes[b % 32] = lanes[b % 32] + a[b]
    total = lanes[0]
    for lane in range(1, 32):
        total = total + lanes[lane]
    return total


def safe_dual_bound_batch(cp, ci, cx, c, row_lb, row_ub, col_lb, col_ub, Y, sum_rows=sum_rows):
    """Valid lower bounds of every node from its dual iterate (safebound.py:194-235)."""
    aty = po.spmm(cp, ci, cx, Y)
    d = c[:, None] - aty
    ru_inf = (row_ub >= INF)[:, None]
    rl_inf = (row_lb <= -INF)[:, None]
    ypos = Y > 0.0
    row_bad = np.where(ypos, rl_inf, ru_inf) & (Y != 0.0)
    row_pick = np.where(ypos, row_lb[:, None], row_ub[:, None])
    row_contrib = np.where(row_bad, 0.0, Y * np.where(row_bad, 0.0, row_pick))
    row_vacuous = row_bad.any(axis=0)
    dpos = d > 0.0
    col_bad = np.where(dpos, col_lb <= -INF, col_ub >= INF) & (d != 0.0)
    col_pick = np.where(dpos, col_lb, col_ub)
    col_contrib = np.where(col_bad, 0.0, d * np.where(col_bad, 0.0, col_pick))
    col_vacuous = col_bad.any(axis=0)
    bounds = sum_rows(row_contrib) + sum_rows(col_contrib)
    return np.where(row_vacuous | col_vacuous, -np.inf, bounds)


class BNROracle:
    """The engine state of ``BNREngine``: the shared scaled problem, and the
    per-node iterates and step sizes that persist between ``solve_batch``
    calls (bnr.py:128-171)."""

    def __init__(self, rp, ri, rx, cp, ci, cx, c, row_lb, row_ub, obj_scale, obj_offset,
                 batch, iters=60, step_growth=0.3, step_damp=0.6, sum_order="sequential"):
        f = lambda a, t=np.float64: np.ascontiguousarray(a, dtype=t)  # noqa: E731
        self.rp, self.ri, self.rx = f(rp, np.int64), f(ri, np.int32), f(rx)
        self.cp, self.ci, self.cx = f(cp, np.int64), f(ci, np.int32), f(cx)
        self.c, self.rl, self.ru = f(c), f(row_lb), f(row_ub)
        self.m, self.n = self.rl.shape[0], self.c.shape[0]
        self.obj_scale = float(obj_scale) or 1.0
        self.obj_offset = float(obj_offset)
        self.iters, self.growth, self.damp = int(iters), float(step_growth), float(step_damp)
        self.sum_rows = {"sequential": sum_rows, "tree": sum_rows_tree}[sum_order]
        self.K = 0
        self._alloc(batch)

    def _alloc(self, K):
        self.K = K
        self.X = np.zeros((self.n, K))
        self.Y = np.zeros((self.m, K))
        self.eta = np.ones(K)
        self.omega = np.ones(K)

    def solve_batch(self, col_lb, col_ub, warm=None):
        """bnr.py:176-301."""
        n, m = self.n, self.m
        L = np.asarray(col_lb, dtype=np.float64)
        U = np.asarray(col_ub, dtype=np.float64)
        K = L.shape[1]
        if K > self.K:
            self._alloc(max(K, self.K * 2))
        empty = (L > U + 1e-12).any(axis=0)
        if warm is not None:
            X = np.array(warm[0], dtype=np.float64)
            Y = np.array(warm[1], dtype=np.float64)
        else:
            X = np.zeros((n, K))
            Y = np.zeros((m, K))
        np.clip(X, L, U, out=X)
        AX = po.spmm(self.rp, self.ri, self.rx, X)
        AtY = po.spmm(self.cp, self.ci, self.cx, Y)
        eta = self.eta[:K].copy()
        omega = self.omega[:K].copy()
        rl_b, ru_b, c_b = self.rl[:, None], self.ru[:, None], self.c[:, None]
        attempts = 0
        for _ in range(self.iters):
            attempts += 1
            tau = (eta / omega)[None, :]
            sigma = (eta * omega)[None, :]
            Xn = np.subtract(X, tau * (c_b + AtY))
            np.clip(Xn, L, U, out=Xn)
            dX = Xn - X
            AdX = po.spmm(self.rp, self.ri, self.rx, dX)
            W = Y + sigma * (AX + 2.0 * AdX)
            Yn = np.subtract(W, sigma * np.clip(W / sigma, rl_b, ru_b))
            dY = Yn - Y
            AtdY = po.spmm(self.cp, self.ci, self.cx, dY)
            S = self.sum_rows
            interaction = np.abs(S(dY * AdX))
            movement = 0.5 * (omega * S(dX * dX) + S(dY * dY) / omega)
            floor = np.maximum(movement, 1.0) / QUOTIENT_MAX
            with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
                limit = np.where(interaction > 0.0, movement / np.maximum(interaction, floor),
                                 np.inf)
            accept = (eta <= limit) | (movement == 0.0)
            a = accept[None, :]
            X = np.where(a, Xn, X)
            Y = np.where(a, Yn, Y)
            AX = np.where(a, AX + AdX, AX)
            AtY = np.where(a, AtY + AtdY, AtY)
            t = attempts + 1
            with np.errstate(invalid="ignore", over="ignore"):
                eta = np.minimum((1.0 - t ** -self.growth) * limit, (1.0 + t ** -self.damp) * eta)
            eta = np.maximum(np.where(np.isfinite(eta), eta, 1.0), 1e-14)
        self.X[:, :K] = X
        self.Y[:, :K] = Y
        self.eta[:K] = eta
        self.omega[:K] = omega
        bounds = safe_dual_bound_batch(self.cp, self.ci, self.cx, self.c, self.rl, self.ru,
                                       L, U, Y, sum_rows=self.sum_rows)
        bounds = (bounds + self.obj_offset) / self.obj_scale
        bounds = np.where(empty, np.inf, bounds)
        return SimpleNamespace(bounds=bounds, x=X.copy(), y=Y.copy(), iterations=self.iters,
                               infeasible=empty)
