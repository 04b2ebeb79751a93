"""Batched node relaxation on the B200 against the reference.

``tests/golden/bnr/*.npz`` hold the reference ``BNREngine``'s outputs for two
consecutive ``solve_batch`` calls (the second continues the first call's step
sizes); ``oracle/bnr_oracle.py`` reproduces them bit for bit.  The device
engine makes the same element-wise operations in the same order and sums each
node's inner products over rows in a fixed tree order, which the oracle
restates as ``sum_order="tree"``:

* the device results equal the tree-order oracle's bit for bit (bounds,
  iterates, step sizes, infeasible flags), on the goldens, with warm starts
  and across the engine's growth;
* against the reference itself they agree to the summation drift that
  ``tests/test_bnr_cpu.py`` bounds: bounds within 1e-9 relative after both
  calls.

Size-independent properties, at sizes beyond the goldens:
* a node's result does not depend on the batch around it (each node solved
  alone gives the same bits as inside a batch of 64);
* the step sizes persist across calls and restart at 1 when the engine grows.
"""

import os
from types import SimpleNamespace

import numpy as np
import pytest

from oracle.bnr_oracle import BNROracle
from sovereign_moe_b200.bnr import BNRConfig, BNREngine
from sovereign_moe_b200.problem import SparseMatrix

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bnr")
CASES = ["bnr_small_s3", "bnr_batch_s11"]
RTOL = 1e-9


def load(name):
    return dict(np.load(os.path.join(HERE, f"{name}.npz")))


def scaled_problem(g):
    A = SparseMatrix(int(g["m"]), int(g["n"]), g["cp"], g["ci"], g["cx"],
                     rp=g["rp"], ri=g["ri"], rx=g["rx"])
    prob = SimpleNamespace(A=A, c=g["c"], row_lb=g["row_lb"], row_ub=g["row_ub"],
                           col_lb=g["col_lb"], col_ub=g["col_ub"],
                           obj_offset=float(g["obj_offset"]))
    return prob, SimpleNamespace(obj=float(g["obj_scale"]))


def engine(g, batch=None, iters=None):
    prob, sc = scaled_problem(g)
    return BNREngine(prob, sc, BNRConfig(batch=batch or int(g["K"]),
                                         iters=int(g["iters"]) if iters is None else iters,
                                         device="gpu"))


def oracle(g, batch=None, iters=None):
    return BNROracle(g["rp"], g["ri"], g["rx"], g["cp"], g["ci"], g["cx"], g["c"],
                     g["row_lb"], g["row_ub"], float(g["obj_scale"]), float(g["obj_offset"]),
                     batch=batch or int(g["K"]),
                     iters=int(g["iters"]) if iters is None else iters, sum_order="tree")


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    assert not bad.any(), (int(bad.sum()), float(np.abs(a - b)[bad].max()))


def close(a, b, rtol=RTOL):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    assert np.array_equal(a[~fin], b[~fin])
    scale = max(1.0, float(np.abs(b[fin]).max(initial=0.0)))
    err = float(np.abs(a[fin] - b[fin]).max(initial=0.0)) / scale
    assert err <= rtol, err


@pytest.mark.parametrize("name", CASES)
def test_two_calls_match_oracle_bitwise(require_gpu, name):
    g = load(name)
    e, o = engine(g), oracle(g)
    K = int(g["K"])
    for call in (1, 2):
        L, U = g[f"L{call}"], g[f"U{call}"]
        r, ro = e.solve_batch(L, U), o.solve_batch(L, U)
        assert np.array_equal(r.infeasible, ro.infeasible)
        assert np.array_equal(r.infeasible, g[f"inf{call}"])
        same(r.bounds, ro.bounds)
        same(r.x, ro.x)
        same(r.y, ro.y)
        same(e.step_sizes(K)[0], o.eta[:K])
        # and the reference's own bounds, to the summation drift
        close(r.bounds, g[f"bounds{call}"])
    assert e.Y is r.y
    st = e.stats()
    assert st["batches"] == 2 and st["nodes_bounded"] == 2 * K
    assert st["pdhg_iterations"] == 2 * int(g["iters"])


def test_empty_node_is_infeasible_with_infinite_bound(require_gpu):
    g = load("bnr_small_s3")
    r = engine(g).solve_batch(g["L1"], g["U1"])
    assert r.infeasible.sum() == 1 and r.infeasible[5]
    assert r.bounds[5] == np.inf
    assert np.isfinite(r.bounds[~r.infeasible]).all()


@pytest.mark.parametrize("name", CASES)
def test_warm_start_matches_oracle(require_gpu, name):
    g = load(name)
    K = int(g["K"])
    rng = np.random.default_rng(5)
    wx = np.asarray(g["x1"]) + 0.01 * rng.standard_normal((int(g["n"]), K))
    wy = np.asarray(g["y1"]) + 0.01 * rng.standard_normal((int(g["m"]), K))
    e, o = engine(g, iters=25), oracle(g, iters=25)
    r = e.solve_batch(g["L2"], g["U2"], warm=(wx, wy))
    ro = o.solve_batch(g["L2"], g["U2"], warm=(wx, wy))
    same(r.bounds, ro.bounds)
    same(r.x, ro.x)
    same(r.y, ro.y)
    same(e.step_sizes(K)[0], o.eta[:K])


def test_growth_restarts_step_sizes_like_the_reference(require_gpu):
    """A batch larger than the engine's capacity doubles it and restarts every
    step size at 1 (bnr.py:149-171); a smaller batch keeps them."""
    g = load("bnr_batch_s11")
    K = int(g["K"])
    e, o = engine(g, batch=K // 2), oracle(g, batch=K // 2)
    half_L, half_U = g["L1"][:, : K // 2], g["U1"][:, : K // 2]
    for L, U in ((half_L, half_U), (g["L1"], g["U1"]), (half_L, half_U)):
        r = e.solve_batch(L, U)
        ro = o.solve_batch(L, U)
        same(r.bounds, ro.bounds)
        same(r.x, ro.x)
        k = L.shape[1]
        same(e.step_sizes(k)[0], o.eta[:k])


def test_node_result_does_not_depend_on_its_batch(require_gpu):
    """64 nodes in one batch against each node alone in a fresh engine: the
    same bits (every product and sum of a node is computed in the same order
    whatever K is)."""
    from sovereign_moe_b200 import workloads
    p = workloads.uneven_batch(seed=4, count=1)[0].problem
    A = p.A
    n = A.n
    lo = np.where(np.isfinite(p.col_lb), p.col_lb, -1e30)
    hi = np.where(np.isfinite(p.col_ub), p.col_ub, 1e30)
    prob = SimpleNamespace(A=A, c=np.asarray(p.c), row_lb=np.asarray(p.row_lb),
                           row_ub=np.asarray(p.row_ub), obj_offset=0.0)
    K = 64
    rng = np.random.default_rng(9)
    L = np.repeat(lo[:, None], K, axis=1)
    U = np.repeat(hi[:, None], K, axis=1)
    boxed = np.flatnonzero((lo > -1e30) & (hi < 1e30) & (hi > lo))
    for k in range(K):
        j = rng.choice(boxed, size=4, replace=False)
        U[j, k] = 0.5 * (lo[j] + hi[j])
    cfg = BNRConfig(batch=K, iters=30, device="gpu")
    rb = BNREngine(prob, SimpleNamespace(obj=1.0), cfg).solve_batch(L, U)
    for k in (0, 17, 63):
        one = BNREngine(prob, SimpleNamespace(obj=1.0), BNRConfig(batch=1, iters=30, device="gpu"))
        r1 = one.solve_batch(L[:, k:k + 1], U[:, k:k + 1])
        assert r1.bounds[0] == rb.bounds[k]
        assert np.array_equal(r1.x[:, 0], rb.x[:, k])
        assert np.array_equal(r1.y[:, 0], rb.y[:, k])
    assert n == rb.x.shape[0]


def test_arguments_are_checked(require_gpu):
    g = load("bnr_small_s3")
    e = engine(g)
    with pytest.raises(ValueError):
        e.solve_batch(g["L1"][:-1], g["U1"][:-1])
    with pytest.raises(ValueError):
        e.solve_batch(g["L1"], g["U1"], warm=(g["x1"], g["y1"][:-1]))
    prob, sc = scaled_problem(g)
    with pytest.raises(ValueError):
        BNREngine(prob, sc, BNRConfig(device="cpu"))


def test_ragged_node_tile_and_tiny_problem(require_gpu):
    """K = 33 (one full 32-node tile and one node in the next) on a golden
    problem, and a 1-row, 3-column LP, each bitwise the tree-order oracle."""
    g = load("bnr_batch_s11")
    rng = np.random.default_rng(33)
    K = 33
    cols = rng.integers(0, int(g["K"]), K)
    L, U = g["L2"][:, cols], g["U2"][:, cols]
    e, o = engine(g, batch=K, iters=20), oracle(g, batch=K, iters=20)
    r, ro = e.solve_batch(L, U), o.solve_batch(L, U)
    same(r.bounds, ro.bounds)
    same(r.x, ro.x)
    same(r.y, ro.y)

    A = SparseMatrix.from_dense(np.array([[1.0, 2.0, -1.0]]))
    prob = SimpleNamespace(A=A, c=np.array([1.0, -1.0, 0.5]), row_lb=np.array([1.0]),
                           row_ub=np.array([1.0]), obj_offset=0.25)
    L = np.zeros((3, 2))
    U = np.array([[1.0, 1.0], [1.0, 0.5], [2.0, 2.0]])
    e = BNREngine(prob, SimpleNamespace(obj=2.0), BNRConfig(batch=2, iters=40, device="gpu"))
    o = BNROracle(A.rp, A.ri, A.rx, A.cp, A.ci, A.cx, prob.c, prob.row_lb, prob.row_ub, 2.0,
                  0.25, batch=2, iters=40, sum_order="tree")
    r, ro = e.solve_batch(L, U), o.solve_batch(L, U)
    same(r.bounds, ro.bounds)
    same(r.x, ro.x)
    same(r.y, ro.y)
    assert np.isfinite(r.bounds).all()


def test_device_pointers_give_the_host_results(require_gpu):
    """The C entry point with device-resident bound sets and outputs
    (PDLP_MEM_DEVICE) returns the same bits as with host arrays."""
    import torch
    from sovereign_moe_b200 import _lib
    g = load("bnr_batch_s11")
    K = int(g["K"])
    e_host, e_dev = engine(g), engine(g)
    r = e_host.solve_batch(g["L1"], g["U1"])
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    dL, dU = dev(g["L1"]), dev(g["U1"])
    db = torch.empty(K, dtype=torch.float64, device="cuda")
    dx = torch.empty((int(g["n"]), K), dtype=torch.float64, device="cuda")
    dy = torch.empty((int(g["m"]), K), dtype=torch.float64, device="cuda")
    dinf = torch.empty(K, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    _lib.check(e_dev.lib.pdlp_bnr_solve_batch(
        e_dev.h, K, dL.data_ptr(), dU.data_ptr(), None, None, int(g["iters"]), 0.3, 0.6,
        db.data_ptr(), dx.data_ptr(), dy.data_ptr(), dinf.data_ptr(), _lib.PDLP_MEM_DEVICE))
    same(db.cpu().numpy(), r.bounds)
    same(dx.cpu().numpy(), r.x)
    same(dy.cpu().numpy(), r.y)
    assert np.array_equal(dinf.cpu().numpy().astype(bool), r.infeasible)


def test_zero_iterations_bound_the_starting_point(require_gpu):
    """iters = 0: the bound of each node's (clipped) warm start, as the
    oracle computes it."""
    g = load("bnr_small_s3")
    e, o = engine(g, iters=0), oracle(g, iters=0)
    warm = (np.asarray(g["x1"]), np.asarray(g["y1"]))
    r, ro = e.solve_batch(g["L2"], g["U2"], warm=warm), o.solve_batch(g["L2"], g["U2"], warm=warm)
    same(r.bounds, ro.bounds)
    same(r.x, ro.x)
    same(r.y, ro.y)


def test_c_entry_point_refuses_bad_arguments(require_gpu):
    from sovereign_moe_b200 import _lib
    g = load("bnr_small_s3")
    e = engine(g)
    L = np.ascontiguousarray(g["L1"])
    U = np.ascontiguousarray(g["U1"])
    x = np.empty((int(g["n"]), 1))
    call = lambda K, iters, wx=None, wy=None, mem=_lib.PDLP_MEM_HOST: e.lib.pdlp_bnr_solve_batch(  # noqa: E731
        e.h, K, L.ctypes.data, U.ctypes.data, wx, wy, iters, 0.3, 0.6, None, None, None, None, mem)
    assert call(0, 10) == _lib.PDLP_ERR_ARG
    assert call(1, -1) == _lib.PDLP_ERR_ARG
    assert call(1, 10, wx=x.ctypes.data) == _lib.PDLP_ERR_ARG
    assert call(1, 10, mem=7) == _lib.PDLP_ERR_ARG
    assert e.lib.pdlp_bnr_step_sizes(e.h, 1 << 20, None, None) == _lib.PDLP_ERR_ARG
    # the engine still works after the refusals
    r = e.solve_batch(g["L1"], g["U1"])
    assert np.isfinite(r.bounds[~r.infeasible]).all()
