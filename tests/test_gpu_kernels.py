"""Kernel-level parity: the Backend entry points of libpdlp_b200.so against the
CPU oracle (the reference's sequential kernels restated in oracle/).

Mirrors the reference's tests/test_gpu.py:78-247 -- SpMV at rtol 1e-12,
row lengths 0/1/31/32/33 under a poisoned output, SpMM across the 32-lane
tile, bitwise-repeatable SpMV, the float32 kernel at 1e-4, the step kernels
at 1e-13 and the reductions at 1e-12 -- called through the C ABI.
"""

import numpy as np
import pytest

from oracle import pdlp_oracle as po
from sovereign_moe_b200.problem import SparseMatrix

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bk(require_gpu):
    from sovereign_moe_b200.backend import get_backend
    return get_backend("gpu")


def _random_csr(m, n, per_col, seed):
    rng = np.random.default_rng(seed)
    cols = np.repeat(np.arange(n), per_col)
    rows = rng.integers(0, m, cols.size)
    vals = rng.standard_normal(cols.size)
    return SparseMatrix.from_triplets(rows, cols, vals, m, n), rng


def _dev(bk, A):
    return bk.pointer(A.rp), bk.index(A.ri), bk.to_device(A.rx)


def test_selftest_known_answer(bk):
    from sovereign_moe_b200.backend import gpu_selftest
    assert gpu_selftest() == (True, None)


@pytest.mark.parametrize("shape", [(400, 600, 5), (3000, 1000, 12), (50, 4000, 3)])
def test_spmv_matches_oracle(bk, shape):
    A, rng = _random_csr(*shape, seed=1)
    x = rng.standard_normal(A.n)
    out = bk.zeros(A.m)
    bk.spmv(*_dev(bk, A), bk.to_device(x), out, A.m)
    bk.sync()
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    np.testing.assert_allclose(bk.to_host(out), exp, rtol=1e-12, atol=1e-12)
    # A^T y through the CSC arrays, as the reference does
    y = rng.standard_normal(A.m)
    outt = bk.zeros(A.n)
    bk.spmv(bk.pointer(A.cp), bk.index(A.ci), bk.to_device(A.cx), bk.to_device(y), outt, A.n)
    bk.sync()
    np.testing.assert_allclose(bk.to_host(outt), po.spmv(A.cp, A.ci, A.cx, y),
                               rtol=1e-12, atol=1e-12)


def test_spmv_handles_empty_and_warp_boundary_rows(bk):
    lens = [0, 1, 31, 32, 33, 0, 64, 65]
    m, n = len(lens), 128
    rng = np.random.default_rng(2)
    rows, cols, vals = [], [], []
    for i, length in enumerate(lens):
        c = rng.choice(n, size=length, replace=False)
        rows += [i] * length
        cols += list(c)
        vals += list(rng.standard_normal(length))
    A = SparseMatrix.from_triplets(np.array(rows), np.array(cols), np.array(vals), m, n)
    x = rng.standard_normal(n)
    out = bk.zeros(m) + 12345.0          # poison: a skipped row is caught
    bk.spmv(*_dev(bk, A), bk.to_device(x), out, m)
    bk.sync()
    np.testing.assert_allclose(bk.to_host(out), po.spmv(A.rp, A.ri, A.rx, x),
                               rtol=1e-12, atol=1e-12)


def test_spmv_long_rows_and_partial_row_blocks(bk):
    """Rows longer than one 128-entry chunk, empty rows between them, and a
    last block of fewer than 32 rows, in both value types."""
    rng = np.random.default_rng(4)
    lens = rng.choice([0, 1, 5, 31, 32, 33, 127, 128, 129, 300, 1000], size=77)
    m, n = len(lens), 1500
    rows = np.repeat(np.arange(m), lens)
    cols = np.concatenate([rng.choice(n, size=k, replace=False) for k in lens])
    A = SparseMatrix.from_triplets(rows, cols, rng.standard_normal(rows.size), m, n)
    x = rng.standard_normal(n)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    out = bk.zeros(m) + 12345.0
    bk.spmv(*_dev(bk, A), bk.to_device(x), out, m)
    bk.sync()
    np.testing.assert_allclose(bk.to_host(out), exp, rtol=1e-12, atol=1e-12)
    import torch
    out32 = torch.full((m,), 12345.0, dtype=torch.float32, device="cuda")
    bk.spmv(bk.pointer(A.rp), bk.index(A.ri), bk.to_device(A.rx).float(),
            bk.to_device(x).float(), out32, m)
    bk.sync()
    np.testing.assert_allclose(out32.cpu().numpy(), exp, rtol=1e-4, atol=1e-3)


def _spmv_ex(bk, variant, A, x, poison=12345.0, f32=False):
    import ctypes
    import torch
    from sovereign_moe_b200 import _lib
    dt = torch.float32 if f32 else torch.float64
    rp, ri = bk.pointer(A.rp), bk.index(A.ri)
    rx = bk.to_device(A.rx).to(dt)
    xd = bk.to_device(x).to(dt)
    out = torch.full((A.m,), poison, dtype=dt, device="cuda")
    fn = bk.lib.pdlp_spmv_ex_f32 if f32 else bk.lib.pdlp_spmv_ex_f64
    _lib.check(fn(variant, A.m, rp.data_ptr(), ri.data_ptr(), rx.data_ptr(), xd.data_ptr(),
                  out.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    bk.sync()
    return out.cpu().numpy()


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_spmv_variants_match_oracle(bk, variant):
    """Every row-block variant (streamed runs of rows, row groups, banded) on
    rows of every length class: empty, short, up to the staging buffer, long
    (the second launch), and blocks that split into several runs.
    The 2000 columns fit the banded variant's shared-memory band."""
    rng = np.random.default_rng(40 + variant)
    lens = rng.choice([0, 1, 3, 7, 8, 9, 15, 16, 17, 40, 100, 255, 256, 257, 600], size=203)
    m, n = len(lens), 2000
    rows = np.repeat(np.arange(m), lens)
    cols = np.concatenate([rng.choice(n, size=k, replace=False) for k in lens])
    A = SparseMatrix.from_triplets(rows, cols, rng.standard_normal(rows.size), m, n)
    x = rng.standard_normal(n)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    np.testing.assert_allclose(_spmv_ex(bk, variant, A, x), exp, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(_spmv_ex(bk, variant, A, x, f32=True), exp, rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("variant", [1, 3])
def test_streamed_rows_equal_oracle_bitwise(bk, variant):
    """Rows of at most 16 entries are always streamed (every 16-row half fits
    the 256-entry buffer), and a streamed row is the oracle's storage-order
    sum of rounded products, bit for bit, whether x is gathered from global
    memory or from the banded variant's shared-memory copy."""
    A, rng = _random_csr(5000, 3000, 4, seed=9)          # about 2.4 entries per row
    lens = np.diff(A.rp)
    assert lens.max() <= 16
    x = rng.standard_normal(A.n)
    got = _spmv_ex(bk, variant, A, x)
    assert np.array_equal(got, po.spmv(A.rp, A.ri, A.rx, x))


@pytest.mark.parametrize("variant", [1, 2, 3])
def test_spmv_rows_summed_in_place_and_by_the_second_launch(bk, variant):
    """Rows of more than 256 entries are summed by the second launch from a
    list kept per stream; rows at and around that bound and far beyond it,
    beside short and empty rows, twice in a row on the same stream."""
    rng = np.random.default_rng(60 + variant)
    lens = [0, 4096, 4097, 9000, 5, 300, 257, 0, 12_000, 3] * 3
    m, n = len(lens), 15_000
    rows = np.repeat(np.arange(m), lens)
    cols = np.concatenate([rng.choice(n, size=k, replace=False) for k in lens])
    A = SparseMatrix.from_triplets(rows, cols, rng.standard_normal(rows.size), m, n)
    for seed in (0, 1):
        x = np.random.default_rng(seed).standard_normal(n)
        exp = po.spmv(A.rp, A.ri, A.rx, x)
        np.testing.assert_allclose(_spmv_ex(bk, variant, A, x), exp, rtol=1e-12, atol=1e-12)


def test_banded_variant_on_a_band_wider_than_shared_memory(bk):
    """Blocks whose index span exceeds the band gather from global memory;
    a banded matrix whose blocks fit stages them; both agree with the oracle."""
    from sovereign_moe_b200.workloads import blending_plan
    wide, rng = _random_csr(20_000, 100_000, 1, seed=13)  # 5 per row; spans far beyond 3072
    x = rng.standard_normal(wide.n)
    np.testing.assert_allclose(_spmv_ex(bk, 3, wide, x), po.spmv(wide.rp, wide.ri, wide.rx, x),
                               rtol=1e-12, atol=1e-12)
    A = blending_plan(seed=1, m=20_000, n=60_000, periods=72, coupling=10).problem.A
    x = rng.standard_normal(A.n)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    np.testing.assert_allclose(_spmv_ex(bk, 3, A, x), exp, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(_spmv_ex(bk, 3, A, x, f32=True), exp, rtol=1e-4, atol=1e-2)


def test_spmv_tuner_and_autotuned_backend(bk):
    import ctypes
    import torch
    from sovereign_moe_b200 import _lib
    from sovereign_moe_b200.backend import Backend
    A, rng = _random_csr(4000, 9000, 6, seed=12)
    x = rng.standard_normal(A.n)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    rp, ri, rx, xd = bk.pointer(A.rp), bk.index(A.ri), bk.to_device(A.rx), bk.to_device(x)
    out = bk.zeros(A.m) + 12345.0
    best = ctypes.c_int32(-1)
    ms = (ctypes.c_double * 3)()
    _lib.check(bk.lib.pdlp_spmv_tune_f64(A.m, rp.data_ptr(), ri.data_ptr(), rx.data_ptr(),
                                         xd.data_ptr(), out.data_ptr(),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                         5, ctypes.byref(best), ms))
    assert best.value in (_lib.PDLP_SPMV_STREAMED, _lib.PDLP_SPMV_ROW_GROUPS,
                          _lib.PDLP_SPMV_BANDED)
    assert min(ms) > 0
    assert ms[best.value - 1] == min(ms)
    np.testing.assert_allclose(out.cpu().numpy(), exp, rtol=1e-12, atol=1e-12)
    tuned = Backend("gpu", autotune=True)
    for _ in range(2):                                   # tunes, then uses the choice
        o = tuned.zeros(A.m) + 12345.0
        tuned.spmv(rp, ri, rx, xd, o, A.m)
        tuned.sync()
        np.testing.assert_allclose(o.cpu().numpy(), exp, rtol=1e-12, atol=1e-12)
    assert len(tuned._spmv_variant) == 1


@pytest.mark.parametrize("k", [1, 8, 32, 33, 64])
def test_spmm_matches_oracle(bk, k):
    A, rng = _random_csr(300, 500, 4, seed=k)
    X = rng.standard_normal((A.n, k))
    Y = bk.zeros((A.m, k))
    bk.spmm(*_dev(bk, A), bk.to_device(X), Y, A.m, k)
    bk.sync()
    np.testing.assert_allclose(bk.to_host(Y), po.spmm(A.rp, A.ri, A.rx, X),
                               rtol=1e-12, atol=1e-12)


def test_spmv_is_bitwise_reproducible(bk):
    A, rng = _random_csr(500, 700, 6, seed=3)
    x = rng.standard_normal(A.n)
    dev, xd = _dev(bk, A), bk.to_device(x)
    first = None
    for _ in range(4):
        out = bk.zeros(A.m)
        bk.spmv(*dev, xd, out, A.m)
        bk.sync()
        got = bk.to_host(out)
        if first is None:
            first = got
        else:
            assert np.array_equal(got, first)


def test_float32_kernel(bk):
    import torch
    A, rng = _random_csr(200, 300, 4, seed=4)
    x = rng.standard_normal(A.n)
    out = torch.zeros(A.m, dtype=torch.float32, device="cuda")
    bk.spmv(bk.pointer(A.rp), bk.index(A.ri),
            torch.as_tensor(A.rx, dtype=torch.float32, device="cuda"),
            torch.as_tensor(x, dtype=torch.float32, device="cuda"), out, A.m)
    bk.sync()
    assert out.dtype == torch.float32
    np.testing.assert_allclose(out.cpu().numpy(), po.spmv(A.rp, A.ri, A.rx, x),
                               rtol=1e-4, atol=1e-4)


def test_primal_and_dual_steps_match_reference_formula(bk):
    rng = np.random.default_rng(5)
    n, m = 1000, 700
    x, c, aty = (rng.standard_normal(n) for _ in range(3))
    lo, hi = -np.abs(rng.standard_normal(n)), np.abs(rng.standard_normal(n))
    y, ax = rng.standard_normal(m), rng.standard_normal(m)
    rl, ru = -np.abs(rng.standard_normal(m)), np.abs(rng.standard_normal(m))
    tau, sigma = 0.37, 1.9
    exp_x = np.clip(x - tau * (c + aty), lo, hi)                 # backend.py:406-409
    w = y + sigma * ax
    exp_y = w - sigma * np.clip(w / sigma, rl, ru)               # backend.py:425-428
    got_x = bk.primal_step(bk.zeros(n), *(bk.to_device(v) for v in (x, c, aty, lo, hi)), tau, n)
    got_y = bk.dual_step(bk.zeros(m), *(bk.to_device(v) for v in (y, ax, rl, ru)), sigma, m)
    bk.sync()
    np.testing.assert_allclose(bk.to_host(got_x), exp_x, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(bk.to_host(got_y), exp_y, rtol=1e-13, atol=1e-13)


def test_fused_pdhg_steps_match_reference_formula(bk):
    rng = np.random.default_rng(6)
    n, m = 800, 600
    x0, c, aty = (rng.standard_normal(n) for _ in range(3))
    lo, hi = -np.ones(n), np.ones(n)
    y0, ax0, adx = (rng.standard_normal(m) for _ in range(3))
    rl, ru = -np.ones(m), np.ones(m)
    tau, sigma, eta = 0.25, 1.4, 0.6
    # the reference's NumPy forms (backend.py:443-474)
    ex = x0.copy()
    xnew = np.clip(ex - tau * (c + aty), lo, hi)
    edx = xnew - ex
    ex[...] = xnew
    ey, eax = y0.copy(), ax0.copy()
    eax += adx
    w = ey + sigma * (eax + adx)
    ynew = w - sigma * np.clip(w / sigma, rl, ru)
    edy = ynew - ey
    ey[...] = ynew
    eacc, erun = aty.copy(), np.zeros(n)
    eacc += edx
    erun += eta * ex

    d = lambda v: bk.to_device(v.copy())                  # noqa: E731
    gx, gdx = d(x0), bk.zeros(n)
    bk.pdhg_primal(gx, gdx, d(c), d(aty), d(lo), d(hi), tau, n)
    gy, gdy, gax = d(y0), bk.zeros(m), d(ax0)
    bk.pdhg_dual(gy, gdy, gax, d(adx), d(rl), d(ru), sigma, m)
    gacc, grun = d(aty), bk.zeros(n)
    bk.pdhg_accum(gacc, gdx, grun, gx, eta, n)
    bk.sync()
    for e, g in zip((ex, edx, ey, edy, eax, eacc, erun), (gx, gdx, gy, gdy, gax, gacc, grun)):
        np.testing.assert_allclose(bk.to_host(g), e, rtol=1e-13, atol=1e-13)


def test_reductions(bk):
    rng = np.random.default_rng(7)
    a, b = rng.standard_normal(40960), rng.standard_normal(40960)
    ag, bg = bk.to_device(a), bk.to_device(b)
    assert bk.dot(ag, bg) == pytest.approx(float(np.dot(a, b)), rel=1e-12)
    assert bk.nrm2(ag) == pytest.approx(float(np.linalg.norm(a)), rel=1e-12)
    assert bk.nrm_inf(ag) == float(np.abs(a).max())
    assert bk.nrm_inf(bk.zeros(0)) == 0.0
    # deterministic: repeated calls agree to the bit
    assert bk.dot(ag, bg) == bk.dot(ag, bg)
