"""``pdlp_dot_noalloc``: the dot product that allocates no device memory.

Called through the C ABI on device vectors and compared with ``pdlp_dot``
(the allocating entry point) at the reductions' tolerance, rel 1e-12, on two
calls in a row -- the second on a shorter vector, so stale partial sums that
the first call left in the shared scratch would show.  The file sorts last so
the entry point also runs after every other GPU test in the same process; it
passes alone in a fresh process too.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 28          # the fixed scratch holds partials for 2^28 elements


@pytest.fixture(scope="module")
def lib(require_gpu):
    from sovereign_moe_b200 import _lib
    return _lib.load()


def _call(fn, n, a, b):
    import torch
    out = ctypes.c_double(float("nan"))
    st = torch.cuda.current_stream().cuda_stream
    code = fn(n, a.data_ptr() if a is not None else None,
              b.data_ptr() if b is not None else None, ctypes.byref(out), st)
    return code, out.value


def _vecs(n, seed):
    import torch
    rng = np.random.default_rng(seed)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    return (torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda"),
            float(np.dot(a, b)))


@pytest.mark.parametrize("sizes", [(3 * 16384 + 7, 40960), (1 << 21, 1), (1, 1 << 21)])
def test_two_calls_match_pdlp_dot(lib, sizes):
    for k, n in enumerate(sizes):
        a, b, exact = _vecs(n, seed=11 + k)
        code, got = _call(lib.pdlp_dot_noalloc, n, a, b)
        assert code == 0, lib.pdlp_last_error().decode()
        code, ref = _call(lib.pdlp_dot, n, a, b)
        assert code == 0, lib.pdlp_last_error().decode()
        assert got == pytest.approx(ref, rel=1e-12, abs=1e-12)
        assert got == pytest.approx(exact, rel=1e-12, abs=1e-12)


def test_repeat_is_bitwise_and_empty_is_zero(lib):
    a, b, _ = _vecs(100_003, seed=5)
    first = _call(lib.pdlp_dot_noalloc, 100_003, a, b)
    second = _call(lib.pdlp_dot_noalloc, 100_003, a, b)
    assert first[0] == 0 and first == second
    assert _call(lib.pdlp_dot_noalloc, 0, None, None) == (0, 0.0)


def test_rejects_sizes_beyond_the_scratch(lib):
    from sovereign_moe_b200 import _lib
    code, _ = _call(lib.pdlp_dot_noalloc, LIMIT + 1, None, None)
    assert code == _lib.PDLP_ERR_ARG
    assert "268435456" in lib.pdlp_last_error().decode()
    code, _ = _call(lib.pdlp_dot_noalloc, -1, None, None)
    assert code == _lib.PDLP_ERR_ARG
