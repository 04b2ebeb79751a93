"""Engine control paths on the GPU: continuous batching, block teams, step
budgets, the bounded device waits and the preconditioner.

* An LP's result does not depend on when it joins a running batch, nor on how
  the engine splits the blocks (one team for more than 256 running LPs, one
  team per LP below that): every per-LP sum runs over the LP's own tiles in an
  order fixed at admission.  These tests compare bitwise against the same LP
  solved alone.
* ``pdlp_batch_step(max_steps)`` advances every running LP by exactly
  ``max_steps`` engine steps (or to its end), however the launches split.
* A device-side wait that runs out ends the step with
  ``PDLP_ERR_BARRIER_TIMEOUT`` and the batch then refuses further calls; the
  CUDA context stays usable.  The wait is made to run out by the test hook
  that withholds one block's arrival (a flag nothing sets), under a 50 ms
  limit; nothing faults.
* The device's pow2 scale factors equal the reference's (``scale_problem(
  method="pdlp")``, tests/golden/*.npz) bit for bit.
"""

import numpy as np
import pytest

import golden_cases as gc
from sovereign_moe_b200 import _lib
from sovereign_moe_b200.batch import BatchEngine
from sovereign_moe_b200.pdlp import PDLPParams
from sovereign_moe_b200.problem import Status
from sovereign_moe_b200.workloads import single_small, uneven_batch

pytestmark = pytest.mark.gpu

P6 = PDLPParams(device="gpu", eps_abs=1e-6, eps_rel=1e-6)


def _alone(prob, params=P6):
    with BatchEngine(max_slots=1) as eng:
        return eng.solve_all([prob], params)[0]


def _same(a, b):
    assert a.status == b.status
    assert a.iterations == b.iterations
    assert np.array_equal(a.x, b.x)
    assert np.array_equal(a.y, b.y)
    assert np.array_equal(a.reduced_costs, b.reduced_costs)


def test_lps_admitted_mid_run_equal_alone(require_gpu):
    """Continuous batching: LPs join while others are mid-solve (the teams are
    re-planned at every join) and each result is bitwise the LP alone."""
    probs = [k.problem for k in uneven_batch(seed=7, count=8, m_lo=60, m_hi=900)]
    with BatchEngine(max_slots=8) as eng:
        slots = [eng.admit(p, P6) for p in probs[:3]]
        eng.step(150)
        assert len(eng.statuses()[eng.statuses() == _lib.PDLP_STATUS_RUNNING]) > 0
        slots += [eng.admit(p, P6) for p in probs[3:6]]
        eng.step(150)
        slots += [eng.admit(p, P6) for p in probs[6:]]
        eng.run()
        together = [eng.fetch(s) for s in slots]
    for p, t in zip(probs, together):
        assert t.status == Status.OPTIMAL
        _same(t, _alone(p))


def test_one_team_above_256_running_lps_equals_alone(require_gpu):
    """With more than 256 LPs running, one team of blocks steps them all;
    as they finish the engine switches to one team per LP.  Both paths give
    each LP its alone result."""
    probs = [k.problem for k in uneven_batch(seed=11, count=300, m_lo=50, m_hi=300)]
    with BatchEngine(max_slots=len(probs)) as eng:
        together = eng.solve_all(probs, P6)
    for i in (0, 1, 57, 150, 299):
        assert together[i].status == Status.OPTIMAL
        _same(together[i], _alone(probs[i]))


def test_step_budget_is_exact(require_gpu):
    """300 steps in one call land where three calls of 100 steps do, with
    LPs finishing inside the calls (their teams go idle and the launch ends
    early, so the engine must relaunch for the rest of the budget)."""
    probs = [k.problem for k in uneven_batch(seed=3, count=6, m_lo=50, m_hi=700)]
    probs.append(gc.load("toy")[0])                # finishes within the first call
    slow = PDLPParams(device="gpu", eps_abs=1e-9, eps_rel=1e-9)

    def run(calls, n):
        with BatchEngine(max_slots=len(probs)) as eng:
            slots = [eng.admit(p, slow) for p in probs]
            for _ in range(calls):
                eng.step(n)
            return [eng.poll(s) for s in slots]

    one, three = run(1, 300), run(3, 100)
    for a, b in zip(one, three):
        assert (a.status, a.iterations, a.restarts, a.rejected_steps) == \
               (b.status, b.iterations, b.restarts, b.rejected_steps)
        assert a.step_size == b.step_size and a.primal_weight == b.primal_weight
    assert any(r.status == _lib.PDLP_STATUS_RUNNING for r in one)


def test_barrier_timeout_is_reported_and_the_batch_refuses_later_calls(require_gpu):
    prob = single_small(seed=0).problem            # 24 tiles a side: a team of several blocks
    with BatchEngine(max_slots=2, barrier_timeout_us=50_000, test_withhold_arrival=True) as eng:
        eng.admit(prob, P6)
        with pytest.raises(_lib.PDLPError) as exc:
            eng.step(64)
        assert exc.value.code == _lib.PDLP_ERR_BARRIER_TIMEOUT
        with pytest.raises(_lib.PDLPError) as exc:
            eng.step(64)
        assert exc.value.code == _lib.PDLP_ERR_STATE
        with pytest.raises(_lib.PDLPError) as exc:
            eng.admit(prob, P6)
        assert exc.value.code == _lib.PDLP_ERR_STATE
    # the context is still usable: a fresh batch solves the LP
    s = _alone(prob)
    assert s.status == Status.OPTIMAL


def test_short_barrier_limit_without_the_hook_solves_normally(require_gpu):
    prob = single_small(seed=1).problem
    with BatchEngine(max_slots=1, barrier_timeout_us=200_000) as eng:
        s = eng.solve_all([prob], P6)[0]
    _same(s, _alone(prob))


@pytest.mark.parametrize("name", ["toy", "testprob", "badly_scaled_s0", "badly_scaled_s2",
                                  "dual_regression", "agree", "small_known_s0", "blend_mini"])
def test_scale_factors_equal_reference_bitwise(require_gpu, name):
    prob, exp = gc.load(name)
    with BatchEngine(max_slots=1) as eng:
        slot = eng.admit(prob, PDLPParams(device="gpu", max_iter=64))
        eng.run()
        r, c, s = eng.scaling(slot)
    assert np.array_equal(r, exp.scale_row)
    assert np.array_equal(c, exp.scale_col)
    assert s == float(exp.scale_obj)


def test_scaling_is_refused_while_preconditioning(require_gpu):
    prob, _ = gc.load("agree")
    with BatchEngine(max_slots=1) as eng:
        slot = eng.admit(prob, P6)
        with pytest.raises(_lib.PDLPError) as exc:
            eng.scaling(slot)
        assert exc.value.code == _lib.PDLP_ERR_STATE


def test_server_requests_arriving_mid_run_equal_alone(require_gpu):
    """Requests arrive while others are on the device (real-time arrivals,
    64-step chunks); every served result is bitwise the LP solved alone with
    the server's parameters."""
    from sovereign_moe_b200.serving import Server
    probs = [k.problem for k in uneven_batch(seed=5, count=10, m_lo=80, m_hi=1500)]
    stream = [(0.004 * i, p) for i, p in enumerate(probs)]
    with Server(max_slots=4, chunk_steps=64) as srv:
        done, stats = srv.serve(stream)
        params = srv.params
    assert stats.completed == len(probs) and stats.max_concurrent >= 2
    for req in done:
        assert req.solution.status == Status.OPTIMAL
        _same(req.solution, _alone(probs[req.rid], params))


def test_admit_many_refuses_only_the_bad_lp(require_gpu):
    """Batched admission: a malformed LP (an index out of range, found by the
    device check) and an LP with a NaN cost are refused with their own codes;
    the others are admitted and solve to their alone results."""
    good = [k.problem for k in uneven_batch(seed=21, count=4, m_lo=60, m_hi=600)]
    bad_idx = good[0].copy()
    bad_idx.A.ri[3] = bad_idx.A.n + 5                   # column index out of range
    bad_nan = good[1].copy()
    bad_nan.c[0] = np.nan
    probs = [good[0], bad_idx, good[1], bad_nan, good[2], good[3]]
    with BatchEngine(max_slots=8) as eng:
        slots, codes = eng.admit_many(probs, P6)
        assert codes == [0, _lib.PDLP_ERR_ARG, 0, _lib.PDLP_ERR_NUMERICAL, 0, 0]
        assert slots[1] == -1 and slots[3] == -1 and len({s for s in slots if s >= 0}) == 4
        eng.run()
        got = [eng.fetch(s) for s in slots if s >= 0]
    for p, t in zip([good[0], good[1], good[2], good[3]], got):
        _same(t, _alone(p))


def test_scheduling_hints_change_no_result(require_gpu):
    """Expected-iteration hints resize the block teams (the LPs expected to
    run longest get their blocks first) but every LP's result stays bitwise
    the one without hints."""
    probs = [k.problem for k in uneven_batch(seed=9, count=12, m_lo=80, m_hi=2500)]
    with BatchEngine(max_slots=12) as eng:
        plain = eng.solve_all(probs, P6)
    hints = [50.0 * (i + 1) ** 2 for i in range(len(probs))]     # deliberately uneven
    with BatchEngine(max_slots=12) as eng:
        hinted = eng.solve_all(probs, P6, hints=hints)
    for a, b in zip(plain, hinted):
        _same(a, b)


def test_collect_many_equals_poll_fetch_retire(require_gpu):
    """``pdlp_batch_collect_many`` (results, x, y, d and retirement of many
    finished slots with one synchronisation) gives the same bits as
    ``pdlp_batch_poll`` + ``pdlp_batch_fetch`` per slot, retires the slots so
    their arenas serve later admissions, and refuses a running, free or
    repeated slot before copying anything."""
    import ctypes
    probs = [k.problem for k in uneven_batch(seed=31, count=5, m_lo=60, m_hi=900)]
    with BatchEngine(max_slots=8) as eng:
        slots, codes = eng.admit_many(probs, P6)
        assert codes == [0] * 5
        lib = eng.lib
        n = len(slots)
        arr = (ctypes.c_int32 * n)(*slots)
        assert lib.pdlp_batch_collect_many(eng.h, n, arr, None, None, None, None, None,
                                           _lib.PDLP_MEM_HOST, 0) == _lib.PDLP_ERR_STATE
        eng.run()
        ref = [eng.fetch(s) for s in slots]
        polls = [eng.poll(s) for s in slots]
        xs = [np.full(p.A.n, np.nan) for p in probs]
        ys = [np.full(p.A.m, np.nan) for p in probs]
        ds = [np.full(p.A.n, np.nan) for p in probs]
        ptr = lambda vs: (ctypes.c_void_p * n)(*[v.ctypes.data for v in vs])  # noqa: E731
        twice = (ctypes.c_int32 * 2)(slots[0], slots[0])
        assert lib.pdlp_batch_collect_many(eng.h, 2, twice, None, None, None, None, None,
                                           _lib.PDLP_MEM_HOST, 1) == _lib.PDLP_ERR_ARG
        res = (_lib.Result * n)()
        hs = [np.full(5 * max(eng._meta[s][2], 1), np.nan) for s in slots]
        assert lib.pdlp_batch_collect_many(eng.h, n, arr, res, ptr(xs), ptr(ys), ptr(ds), ptr(hs),
                                           _lib.PDLP_MEM_HOST, 1) == 0
        for i in range(n):
            assert bytes(res[i]) == bytes(polls[i])
            assert np.array_equal(xs[i], ref[i].x) and np.array_equal(ys[i], ref[i].y)
            assert np.array_equal(ds[i], ref[i].reduced_costs)
            hl = res[i].history_len
            assert hl == len(ref[i].log) and np.array_equal(
                hs[i][:5 * hl].reshape(-1, 5), np.array(ref[i].log, dtype=float).reshape(-1, 5))
        # retired: the slots are free, and a new admission reuses an arena
        assert lib.pdlp_batch_collect_many(eng.h, 1, (ctypes.c_int32 * 1)(slots[0]), None, None,
                                           None, None, None, _lib.PDLP_MEM_HOST, 1) == _lib.PDLP_ERR_ARG
        assert list(eng.statuses()[:8]).count(_lib.PDLP_SLOT_FREE) == 8
        again, codes = eng.admit_many(probs[:2], P6)
        assert codes == [0, 0]
        eng.run()
        _same(eng.fetch(again[0]), ref[0])
