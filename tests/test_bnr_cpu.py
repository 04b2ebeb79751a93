"""The BNR oracle against the reference's own outputs.

``tests/golden/bnr/*.npz`` hold what the reference's ``BNREngine`` returned
on its CPU backend for two consecutive ``solve_batch`` calls (the second
continues the first call's step sizes).  The restatement in
``oracle/bnr_oracle.py`` must return the same bounds, iterates, infeasible
flags and step sizes, bit for bit.

The device engine sums each node's inner products over rows in a fixed tree
order (``sum_order="tree"`` in the oracle).  Its results drift from the
reference's by rounding that the step-size test amplifies: the bounds agree
within 1e-9 relative after both calls; the iterates within 1e-9 after the
first call and 1e-6 after the second (measured: 1.5e-7), the step sizes
within 1e-5 (measured: 6.4e-7).
"""

import os

import numpy as np
import pytest

from oracle.bnr_oracle import BNROracle

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bnr")
CASES = ["bnr_small_s3", "bnr_batch_s11"]


def load(name):
    return dict(np.load(os.path.join(HERE, f"{name}.npz")))


def oracle_for(g):
    return BNROracle(g["rp"], g["ri"], g["rx"], g["cp"], g["ci"], g["cx"], g["c"],
                     g["row_lb"], g["row_ub"], float(g["obj_scale"]), float(g["obj_offset"]),
                     batch=int(g["K"]), iters=int(g["iters"]))


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_bnr(name):
    g = load(name)
    o = oracle_for(g)
    r1 = o.solve_batch(g["L1"], g["U1"])
    assert np.array_equal(r1.infeasible, g["inf1"])
    assert np.array_equal(r1.bounds, g["bounds1"])
    assert np.array_equal(r1.x, g["x1"])
    assert np.array_equal(r1.y, g["y1"])
    assert np.array_equal(o.eta[: int(g["K"])], g["eta1"])
    r2 = o.solve_batch(g["L2"], g["U2"])
    assert np.array_equal(r2.bounds, g["bounds2"])
    assert np.array_equal(r2.x, g["x2"])
    assert np.array_equal(r2.y, g["y2"])
    assert np.array_equal(o.eta[: int(g["K"])], g["eta2"])


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    fin = np.isfinite(b)
    assert np.array_equal(a[~fin], b[~fin])
    return float(np.abs(a[fin] - b[fin]).max(initial=0.0)) / max(1.0, float(np.abs(b[fin]).max(initial=0.0)))


@pytest.mark.parametrize("name", CASES)
def test_tree_order_drift_from_reference_is_bounded(name):
    g = load(name)
    o = BNROracle(g["rp"], g["ri"], g["rx"], g["cp"], g["ci"], g["cx"], g["c"],
                  g["row_lb"], g["row_ub"], float(g["obj_scale"]), float(g["obj_offset"]),
                  batch=int(g["K"]), iters=int(g["iters"]), sum_order="tree")
    K = int(g["K"])
    r1 = o.solve_batch(g["L1"], g["U1"])
    assert np.array_equal(r1.infeasible, g["inf1"])
    assert rel(r1.bounds, g["bounds1"]) <= 1e-9
    assert rel(r1.x, g["x1"]) <= 1e-9 and rel(r1.y, g["y1"]) <= 1e-9
    assert rel(o.eta[:K], g["eta1"]) <= 1e-9
    r2 = o.solve_batch(g["L2"], g["U2"])
    assert rel(r2.bounds, g["bounds2"]) <= 1e-9
    assert rel(r2.x, g["x2"]) <= 1e-6 and rel(r2.y, g["y2"]) <= 1e-6
    assert rel(o.eta[:K], g["eta2"]) <= 1e-5


def test_tree_sum_is_the_block_phase_lane_order():
    from oracle.bnr_oracle import sum_rows_tree
    rng = np.random.default_rng(1)
    for rows in (1, 7, 64, 65, 230, 64 * 40 + 3):
        P = rng.standard_normal((rows, 3))
        blocks = []
        for b0 in range(0, rows, 64):
            blk = P[b0:b0 + 64]
            ph = [np.zeros(3) for _ in range(8)]
            for r in range(blk.shape[0]):
                ph[r % 8] = ph[r % 8] + blk[r]
            a = ph[0]
            for y in range(1, 8):
                a = a + ph[y]
            blocks.append(a)
        lanes = [np.zeros(3) for _ in range(32)]
        for b, a in enumerate(blocks):
            lanes[b % 32] = lanes[b % 32] + a
        want = lanes[0]
        for lane in range(1, 32):
            want = want + lanes[lane]
        assert np.array_equal(sum_rows_tree(P), want)


def test_planted_mistake_is_caught():
    """A wrong step-size exponent in the oracle changes the result."""
    g = load("bnr_small_s3")
    o = oracle_for(g)
    o.damp = 0.5
    r1 = o.solve_batch(g["L1"], g["U1"])
    assert not np.array_equal(r1.bounds, g["bounds1"])


def test_node_relaxation_workload_is_a_feasible_node_batch():
    """The bench's node batch: a 20,000 x 30,000 LP with 8 entries per column,
    equality rows met by an interior point of the [0, 10] box, and 128 bound
    sets that each halve the box of 3 columns (a smaller copy here)."""
    from sovereign_moe_b200.workloads import node_relaxation
    prob, L, U = node_relaxation(m=400, n=600, per_col=8, nodes=16)
    A = prob.A
    assert (A.m, A.n) == (400, 600) and A.nnz == 600 * 8
    assert np.array_equal(np.diff(A.cp), np.full(600, 8))
    assert np.array_equal(prob.row_lb, prob.row_ub)
    assert L.shape == U.shape == (600, 16)
    assert ((L == 0) | (L == 5)).all() and ((U == 10) | (U == 5)).all() and (L <= U).all()
    assert ((L != 0) | (U != 10)).sum(axis=0).tolist() == [3] * 16
    # the oracle bounds every node with finite, deterministic values
    o = BNROracle(A.rp, A.ri, A.rx, A.cp, A.ci, A.cx, prob.c, prob.row_lb, prob.row_ub,
                  1.0, 0.0, batch=16, iters=20)
    r = o.solve_batch(L, U)
    assert np.isfinite(r.bounds).all() and not r.infeasible.any()
    r2 = BNROracle(A.rp, A.ri, A.rx, A.cp, A.ci, A.cx, prob.c, prob.row_lb, prob.row_ub,
                   1.0, 0.0, batch=16, iters=20).solve_batch(L, U)
    assert np.array_equal(r.bounds, r2.bounds)


def test_bnr_iteration_bytes():
    """The algorithmic bytes the bnr bench line divides by its time."""
    import bench
    m, n, nnz, K = 20_000, 30_000, 240_000, 128
    assert bench.bnr_bytes_per_iteration(m, n, nnz, K) == (
        8 * (10 * n + 9 * m) * K + 2 * 12 * nnz + 8 * (m + 1) + 8 * (n + 1))


def test_bench_workloads_are_seeded():
    """The bench's synthetic inputs are the same on every machine: the same
    seed gives the same arrays, another seed different ones."""
    from sovereign_moe_b200.workloads import node_relaxation, uneven_batch
    a = uneven_batch(seed=5, count=3, m_lo=50, m_hi=300)
    b = uneven_batch(seed=5, count=3, m_lo=50, m_hi=300)
    c = uneven_batch(seed=6, count=3, m_lo=50, m_hi=300)
    for x, y in zip(a, b):
        assert np.array_equal(x.problem.A.cx, y.problem.A.cx)
        assert np.array_equal(x.problem.c, y.problem.c) and x.f_star == y.f_star
    assert not all(np.array_equal(x.problem.c, z.problem.c) if x.problem.c.shape == z.problem.c.shape
                   else False for x, z in zip(a, c))
    p1, L1, U1 = node_relaxation(m=100, n=150, per_col=4, nodes=4)
    p2, L2, U2 = node_relaxation(m=100, n=150, per_col=4, nodes=4)
    assert np.array_equal(p1.A.cx, p2.A.cx) and np.array_equal(L1, L2) and np.array_equal(U1, U2)
