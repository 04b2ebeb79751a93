"""The engine autotuner on the GPU (``pdlp_tune_lp``, ``autotune`` batches).

The tuner times solo runs of an LP with each candidate lanes-per-row and tile
shape and caches the fastest under the LP's nnz profile.  A batch created with
``autotune`` admits LPs of a cached profile with the tuned choice.  Tuning
changes only how rows are split across lanes and warps, so a tuned solve
reaches the same optimum (objective within 1e-6 of the known one, accepted by
the verifier) and, with the fixed rules' choice, the very same bits.
"""

import ctypes

import numpy as np
import pytest

from oracle import verify_oracle as vo
from sovereign_moe_b200 import _lib, tuning
from sovereign_moe_b200.batch import BatchEngine
from sovereign_moe_b200.pdlp import PDLPParams
from sovereign_moe_b200.problem import Status
from sovereign_moe_b200.workloads import uneven_batch

pytestmark = pytest.mark.gpu

P6 = PDLPParams(device="gpu", eps_abs=1e-6, eps_rel=1e-6)


def test_tuned_batches_reach_the_known_optimum(require_gpu):
    tuning.clear()
    ks = uneven_batch(seed=31, count=6, m_lo=200, m_hi=3000)
    probs = [k.problem for k in ks]
    done = tuning.tune(probs, P6)
    assert len(done) == len({tuning.profile_key(p.A.m, p.A.n, p.A.nnz) for p in probs})
    for t in done.values():
        assert t["lanes_rows"] in (1, 2, 4) and t["lanes_cols"] in (1, 2, 4)
        assert (t["tile_rows"], t["tile_nnz"]) in ((64, 512), (32, 512), (64, 256), (32, 256))
        # the chosen candidate is at least as fast as the fixed rules' (both timed)
        assert 0 < t["us_per_iteration"] <= t["default_us_per_iteration"]
    with BatchEngine(max_slots=8, autotune=True) as eng:
        tuned = eng.solve_all(probs, P6)
    with BatchEngine(max_slots=8) as eng:
        plain = eng.solve_all(probs, P6)
    for k, t, p in zip(ks, tuned, plain):
        assert t.status == p.status == Status.OPTIMAL
        assert abs(t.objective - k.f_star) / max(1.0, abs(k.f_star)) < 1e-6
        assert vo.verify(k.problem, t.x, t.objective, feas_tol=1e-6).ok
    tuning.clear()


def test_a_cached_default_choice_gives_the_same_bits(require_gpu):
    """An entry that holds the fixed rules' own choice changes nothing."""
    k = uneven_batch(seed=33, count=1, m_lo=500, m_hi=600)[0]
    A = k.problem.A
    tuning.clear()
    key = _lib.TuneKey(*tuning.profile_key(A.m, A.n, A.nnz))
    lanes = lambda avg: 1 if avg <= 48 else (2 if avg <= 160 else 4)   # noqa: E731
    t = _lib.Tuning(lanes(A.nnz / A.m), lanes(A.nnz / A.n), 64, 512, 1.0, 1.0)
    _lib.check(_lib.load().pdlp_tune_cache_put(ctypes.byref(key), ctypes.byref(t)))
    with BatchEngine(max_slots=1, autotune=True) as eng:
        a = eng.solve_all([k.problem], P6)[0]
    with BatchEngine(max_slots=1) as eng:
        b = eng.solve_all([k.problem], P6)[0]
    assert a.iterations == b.iterations and np.array_equal(a.x, b.x)
    tuning.clear()
