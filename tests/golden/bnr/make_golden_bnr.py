"""Generate the golden fixtures that pin the batched node relaxation (BNR)
oracle to the reference.

Runs the reference ``sovopt``'s ``BNREngine`` (``src/sovopt/mip/bnr.py``) on
its CPU backend, imported read-only from a checkout, and stores per case:
- the pdlp-scaled problem it was given;
- the per-node column bounds of two consecutive ``solve_batch`` calls (the
  second continues the first call's step sizes, as the reference's engine
  does);
- what each call returned: bounds, x, infeasible flags, the dual iterate Y,
  and the step sizes after the call.

``tests/test_bnr_cpu.py`` replays every case through ``oracle/bnr_oracle.py``.

Usage (needs the reference checkout; not run by the tests):

    SOVOPT_JIT_CACHE=0 PYTHONDONTWRITEBYTECODE=1 \\
        python tests/golden/bnr/make_golden_bnr.py /path/to/Sovereign-MOE
"""

from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))


def node_bounds(lo, hi, K, rng, empty_node=None):
    """K bound sets: node k tightens three random boxed columns to one half of
    their box (a branching-like change); ``empty_node`` gets a crossed box."""
    L = np.repeat(lo[:, None], K, axis=1).copy()
    U = np.repeat(hi[:, None], K, axis=1).copy()
    boxed = np.flatnonzero((lo > -1e30) & (hi < 1e30) & (hi > lo))
    for k in range(K):
        for j in rng.choice(boxed, size=min(3, boxed.size), replace=False):
            mid = 0.5 * (lo[j] + hi[j])
            if rng.random() < 0.5:
                U[j, k] = mid
            else:
                L[j, k] = mid
    if empty_node is not None:
        j = boxed[0]
        L[j, empty_node] = hi[j] + 1.0
    return L, U


def main(ref_root):
    os.environ.setdefault("SOVOPT_JIT_CACHE", "0")
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(ref_root, "src"))
    sys.path.insert(0, REPO)
    from sovopt.core.problem import Problem as RProblem
    from sovopt.core.sparse import SparseMatrix as RSparse
    from sovopt.mip.bnr import BNRConfig, BNREngine
    from sovopt.numerics.scaling import scale_problem
    from sovereign_moe_b200 import workloads

    cases = [("bnr_small_s3", workloads.single_small(seed=3), 12, 5, 60),
             ("bnr_batch_s11", workloads.uneven_batch(seed=11, count=1)[0], 16, None, 40)]
    for name, k, K, empty, iters in cases:
        p = k.problem
        A = p.A
        rows = np.repeat(np.arange(A.m), np.diff(A.rp))
        RA = RSparse.from_triplets(rows, np.asarray(A.ri), np.asarray(A.rx), A.m, A.n)
        rp = RProblem(A=RA, c=np.asarray(p.c), row_lb=np.asarray(p.row_lb),
                      row_ub=np.asarray(p.row_ub), col_lb=np.asarray(p.col_lb),
                      col_ub=np.asarray(p.col_ub))
        scaled, sc = scale_problem(rp, method="pdlp")
        eng = BNREngine(scaled, sc, BNRConfig(batch=K, iters=iters, device="cpu"))
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        L1, U1 = node_bounds(scaled.col_lb, scaled.col_ub, K, rng, empty)
        r1 = eng.solve_batch(L1, U1)
        y1 = np.asarray(eng.Y[:, :K]).copy()
        eta1 = eng.eta[:K].copy()
        L2, U2 = node_bounds(scaled.col_lb, scaled.col_ub, K, rng, None)
        r2 = eng.solve_batch(L2, U2)
        y2 = np.asarray(eng.Y[:, :K]).copy()
        SA = scaled.A
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            m=SA.m, n=SA.n, rp=SA.rp, ri=SA.ri, rx=SA.rx, cp=SA.cp, ci=SA.ci, cx=SA.cx,
            c=scaled.c, row_lb=scaled.row_lb, row_ub=scaled.row_ub,
            col_lb=scaled.col_lb, col_ub=scaled.col_ub, obj_offset=scaled.obj_offset,
            obj_scale=float(getattr(sc, "obj", 1.0) or 1.0), iters=iters, K=K,
            L1=L1, U1=U1, bounds1=r1.bounds, x1=r1.x, inf1=r1.infeasible, y1=y1, eta1=eta1,
            L2=L2, U2=U2, bounds2=r2.bounds, x2=r2.x, inf2=r2.infeasible, y2=y2,
            eta2=eng.eta[:K].copy())
        print(name, "bounds1", np.round(r1.bounds[:4], 6), "inf", r1.infeasible.sum(),
              "bounds2", np.round(r2.bounds[:4], 6))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT  "
                 "(the root of the reference source tree, holding src/sovopt)")
    main(sys.argv[1])
