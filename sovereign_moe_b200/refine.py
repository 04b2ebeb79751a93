"""Mixed precision: float32 PDHG inner solves, float64 outer refinement.

``solve_refined(prob, params, target=1e-8)`` solves the LP by iterative
refinement (Gleixner, Steffy & Wolter, "Iterative refinement for linear
programming", INFORMS J. Computing 28 (2016)).  Each round solves, with the
engine's float32-SpMV PDHG at a loose relative tolerance, the *residual* LP of
the current float64 point (x̄, ȳ):

    min (Δd·d̄)ᵀ x̂   s.t.   A x̂ = Δp·(b − A x̄),   Δp·(l − x̄) ≤ x̂ ≤ Δp·(u − x̄)

with d̄ = c − Aᵀȳ, then corrects x̄ += x̂/Δp, ȳ += ŷ/Δd.  The scale factors Δp,
Δd blow the residual LP back up to unit size, so a loose inner solve gains a
fixed number of digits per round.  Residuals, the corrections and the
termination test run in float64 on the GPU (``Backend`` SpMVs on the device
copy of A); termination uses the reference's test (``src/sovopt/lp/pdlp.py:
523-530``) on the original problem at ``eps_abs = eps_rel = target``.

Rows with ``rl < ru`` get a slack column (``A x − s = 0``, ``rl ≤ s ≤ ru``)
so every residual LP has equality rows; the slacks are dropped on return.
The reference has no refinement step -- its PDLP is float64 throughout.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .batch import BatchEngine
from .pdlp import PDLPParams, PDLPInfo, params_struct
from .problem import INF, ObjSense, Problem, Solution, SparseMatrix, Status

__all__ = ["solve_refined", "equality_form"]


def equality_form(prob):
    """``(A', c', b', l', u', n_orig, flip)``: the LP with a slack column for
    every row whose bounds differ, rows ``A' z = b'`` (b' = rl on equality
    rows, 0 on slack rows), minimisation sense."""
    A = prob.A
    m, n = A.m, A.n
    rl = np.asarray(prob.row_lb, dtype=np.float64)
    ru = np.asarray(prob.row_ub, dtype=np.float64)
    flip = int(prob.sense) == int(ObjSense.MAXIMISE)
    c = -np.asarray(prob.c, dtype=np.float64) if flip else np.asarray(prob.c, dtype=np.float64)
    ineq = np.flatnonzero(rl != ru)
    k = ineq.size
    if k == 0:
        return A, c, rl.copy(), np.asarray(prob.col_lb, float), np.asarray(prob.col_ub, float), n, flip
    cols = np.repeat(np.arange(n), np.diff(A.cp))
    rows = np.concatenate([A.ci.astype(np.int64), ineq])
    cc = np.concatenate([cols, n + np.arange(k)])
    vals = np.concatenate([A.cx, -np.ones(k)])
    A2 = SparseMatrix.from_triplets(rows, cc, vals, m, n + k)
    b = rl.copy()
    b[ineq] = 0.0
    l2 = np.concatenate([prob.col_lb, rl[ineq]])
    u2 = np.concatenate([prob.col_ub, ru[ineq]])
    c2 = np.concatenate([c, np.zeros(k)])
    return A2, c2, b, l2, u2, n, flip


def solve_refined(prob, params: PDLPParams | None = None, target=1e-8, inner_eps=1e-4,
                  max_rounds=12, precision="fp32", growth=1e6):
    """Solve ``prob`` to the reference's KKT test at ``target`` with float32
    inner PDHG solves and float64 refinement on the GPU.  Returns a
    ``Solution`` (``method="pdlp[gpu,refined]"``); ``info.history`` lists
    ``(round, inner iterations, primal violation, gap)``."""
    import torch
    from .backend import Backend

    t0 = time.perf_counter()
    params = params or PDLPParams(device="gpu")
    bk = Backend("gpu")
    A, c, b, lo, hi, n_orig, flip = equality_form(prob)
    m, n = A.m, A.n
    dev = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), device="cuda").to(dt)  # noqa: E731
    rp, ri, rx = dev(A.rp, torch.int64), dev(A.ri, torch.int32), dev(A.rx)
    cp, ci, cx = dev(A.cp, torch.int64), dev(A.ci, torch.int32), dev(A.cx)
    cd, bd, lod, hid = dev(c), dev(b), dev(lo), dev(hi)
    lo_fin, hi_fin = lod > -INF, hid < INF
    v0 = dev(np.random.default_rng(0).standard_normal(n))
    ax = torch.empty(m, dtype=torch.float64, device="cuda")
    aty = torch.empty(n, dtype=torch.float64, device="cuda")

    inner = PDLPParams(**{**params.__dict__})
    inner.eps_abs = inner.eps_rel = inner_eps
    inner.feas_cap = 1e300            # inner tolerance purely relative
    inner.precision = precision
    inner.device = "gpu"

    # reference termination quantities of the ORIGINAL problem (pdlp.py:523-530)
    rl0 = np.asarray(prob.row_lb, float)
    ru0 = np.asarray(prob.row_ub, float)
    rhs = max(float(np.abs(np.where(rl0 > -INF, rl0, 0.0)).max(initial=0.0)),
              float(np.abs(np.where(ru0 < INF, ru0, 0.0)).max(initial=0.0)))
    cn = float(np.abs(np.asarray(prob.c, float)).max(initial=0.0))
    ptol = min(target + target * rhs, params.feas_cap)
    dtol = min(target + target * cn, params.feas_cap)

    eng = BatchEngine(max_slots=1)
    rd = torch.empty(m, dtype=torch.float64, device="cuda")
    cdv = torch.empty(n, dtype=torch.float64, device="cuda")
    lr = torch.empty(n, dtype=torch.float64, device="cuda")
    ur = torch.empty(n, dtype=torch.float64, device="cuda")

    def inner_solve(cvec, rowb, lvec, uvec):
        d = _lib.ProblemDesc()
        d.m, d.n, d.nnz = m, n, int(A.nnz)
        d.rp, d.ri, d.rx = rp.data_ptr(), ri.data_ptr(), rx.data_ptr()
        d.cp, d.ci, d.cx = cp.data_ptr(), ci.data_ptr(), cx.data_ptr()
        d.c = cvec.data_ptr()
        d.row_lb = d.row_ub = rowb.data_ptr()
        d.col_lb, d.col_ub = lvec.data_ptr(), uvec.data_ptr()
        d.kind = None
        d.obj_offset = 0.0
        d.sense = 1
        d.memory = _lib.PDLP_MEM_DEVICE
        p, _ = params_struct(inner, n, power_start=None, history_capacity=0)
        p.power_start = v0.data_ptr()
        slot = ctypes.c_int32(-1)
        _lib.check(eng.lib.pdlp_batch_admit(eng.h, ctypes.byref(d), ctypes.byref(p),
                                            ctypes.byref(slot)))
        eng.run()
        r = eng.poll(slot.value)
        xs = torch.empty(n, dtype=torch.float64, device="cuda")
        ys = torch.empty(m, dtype=torch.float64, device="cuda")
        _lib.check(eng.lib.pdlp_batch_fetch(eng.h, slot.value, xs.data_ptr(), ys.data_ptr(),
                                            None, None, _lib.PDLP_MEM_DEVICE))
        eng.retire(slot.value)
        return xs, ys, int(r.iterations), int(r.status)

    def measures(x, y):
        bk.spmv(rp, ri, rx, x, ax, m)
        bk.spmv(cp, ci, cx, y, aty, n)
        res = bd - ax
        bv = torch.clamp(lod - x, min=0) + torch.clamp(x - hid, min=0)
        pviol = max(float(res.abs().max()) if m else 0.0, float(bv.max()) if n else 0.0)
        dbar = cd - aty
        dres = torch.where(lo_fin, torch.zeros_like(dbar), torch.clamp(dbar, min=0)) + \
            torch.where(hi_fin, torch.zeros_like(dbar), torch.clamp(-dbar, min=0))
        dviol = float(dres.max()) if n else 0.0
        pobj = float(torch.dot(cd, x))
        bnd = torch.where(dbar > 0, torch.where(lo_fin, lod, torch.zeros_like(lod)),
                          torch.where(hi_fin, hid, torch.zeros_like(hid))) * dbar
        dobj = float(torch.dot(bd, y) + bnd.sum())
        return res, dbar, pviol, dviol, pobj, dobj

    history = []
    total_inner = 0
    try:
        x, y, its, st = inner_solve(cd, bd, lod, hid)
        total_inner += its
        dp = dd = 1.0
        status = Status.ITERATION_LIMIT
        for rnd in range(max_rounds + 1):
            res, dbar, pviol, dviol, pobj, dobj = measures(x, y)
            gap = abs(pobj - dobj)
            history.append((rnd, its, pviol, gap))
            if pviol <= ptol and dviol <= dtol and gap <= target + target * (abs(pobj) + abs(dobj)):
                status = Status.OPTIMAL
                break
            if rnd == max_rounds:
                break
            dp = min(1.0 / max(pviol, 1e-300), dp * growth)
            dd = min(1.0 / max(gap / max(1.0, abs(pobj)), dviol, 1e-300), dd * growth)
            torch.mul(res, dp, out=rd)
            torch.mul(dbar, dd, out=cdv)
            torch.where(lo_fin, (lod - x) * dp, lod, out=lr)
            torch.where(hi_fin, (hid - x) * dp, hid, out=ur)
            xh, yh, its, st = inner_solve(cdv, rd, lr, ur)
            total_inner += its
            x = x + xh / dp
            y = y + yh / dd
    finally:
        eng.close()

    xh = x.cpu().numpy()[:n_orig]
    yh = y.cpu().numpy()
    if flip:
        yh = -yh
    xh = np.clip(xh, prob.col_lb, prob.col_ub)
    obj = float(np.asarray(prob.c, float) @ xh) + float(prob.obj_offset)
    d = np.asarray(prob.c, float) - prob.A.rmatvec(yh)
    info = PDLPInfo(iterations=total_inner, device="gpu", history=history)
    sol = Solution(status=status, x=xh, objective=obj, y=yh, reduced_costs=d,
                   iterations=total_inner, time=time.perf_counter() - t0,
                   method="pdlp[gpu,refined]")
    sol.log = history
    sol.dual_bound = obj
    sol.work_units = float(total_inner)
    sol.info = info
    return sol.drop_objective_if_unsolved()
