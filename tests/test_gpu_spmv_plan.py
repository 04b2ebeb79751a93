"""The planned SpMV (``pdlp_spmv_plan_*``) against the CPU oracle.

The oracle is the reference's storage-order CSR product (sparse.py:50-58,
restated in oracle/sparse_ref.c).  Rows of at most 64 entries are summed by
one lane in storage order, so they must equal the oracle bit for bit; longer
rows are summed lane-strided and are checked at the SpMV tolerance of the
reference's GPU tests, rtol 1e-12 (float32 at 1e-4).  Outputs are poisoned
first, so a row the kernel skips is caught.
"""

import ctypes

import numpy as np
import pytest

from oracle import pdlp_oracle as po
from sovereign_moe_b200.problem import SparseMatrix

pytestmark = pytest.mark.gpu

POISON = 12345.0


class Csr:
    """Row pointers, column indices and values of an m x n CSR matrix."""

    def __init__(self, m, n, rp, ri, rx):
        self.m, self.n = int(m), int(n)
        self.rp = np.ascontiguousarray(rp, np.int64)
        self.ri = np.ascontiguousarray(ri, np.int32)
        self.rx = np.ascontiguousarray(rx, np.float64)

    @property
    def nnz(self):
        return int(self.ri.shape[0])

    @classmethod
    def of(cls, A):
        return cls(A.m, A.n, A.rp, A.ri, A.rx)

    @classmethod
    def transpose_of(cls, A):
        return cls(A.n, A.m, A.cp, A.ci, A.cx)


@pytest.fixture(scope="module")
def bk(require_gpu):
    from sovereign_moe_b200.backend import get_backend
    return get_backend("gpu")


def _banded_cols(rng, i, m, n, k, far=0.03):
    """k distinct columns of row i: most in a window that follows the
    diagonal, a few (``far``) anywhere."""
    width = min(n, max(int(k) + 64, 1500))
    lo = min(max(0, int(i * n / max(m, 1)) - width // 2), n - width)
    near = lo + rng.choice(width, size=int(k), replace=False)
    move = rng.random(int(k)) < far
    cand = near.copy()
    cand[move] = rng.integers(0, n, int(move.sum()))
    return cand if np.unique(cand).size == cand.size else near


def _matrix(lens, n, seed, sort=True, banded=False):
    rng = np.random.default_rng(seed)
    m = len(lens)
    rows = np.repeat(np.arange(m), lens)
    if banded:
        cols = np.concatenate([_banded_cols(rng, i, m, n, k) for i, k in enumerate(lens)])
    else:
        cols = np.concatenate([rng.choice(n, size=int(k), replace=False) for k in lens]
                              ) if len(lens) else np.zeros(0, np.int64)
    A = Csr.of(SparseMatrix.from_triplets(rows, cols, rng.standard_normal(rows.size), m, n))
    if not sort:                       # storage order within each row reversed
        ri = A.ri.copy()
        rx = A.rx.copy()
        for i in range(m):
            a, b = A.rp[i], A.rp[i + 1]
            ri[a:b] = ri[a:b][::-1]
            rx[a:b] = rx[a:b][::-1]
        A = Csr(m, n, A.rp, ri, rx)
    return A, rng


def _run(bk, A, x, f32=False, plan=None, poison=POISON):
    import torch
    dt = torch.float32 if f32 else torch.float64
    rp, ri = bk.pointer(A.rp), bk.index(A.ri)
    if plan is None:
        plan = bk.spmv_plan(rp, ri, A.m, A.n)
    out = torch.full((A.m,), poison, dtype=dt, device="cuda")
    bk.spmv_planned(plan, bk.to_device(A.rx).to(dt), bk.to_device(x).to(dt), out)
    assert plan.status(bk._stream()) == 0
    return out.cpu().numpy(), plan


def _short_rows(A, limit=64):
    return np.diff(A.rp) <= limit


@pytest.mark.parametrize("shape", [(400, 600, 5), (3000, 1000, 12), (50, 4000, 3),
                                   (20000, 30000, 6)])
def test_plan_matches_oracle_both_products(bk, shape):
    m, n, per_col = shape
    rng = np.random.default_rng(1)
    cols = np.repeat(np.arange(n), per_col)
    rows = rng.integers(0, m, cols.size)
    S = SparseMatrix.from_triplets(rows, cols, rng.standard_normal(cols.size), m, n)
    A = Csr.of(S)
    x = rng.standard_normal(n)
    got, _ = _run(bk, A, x)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)
    short = _short_rows(A)
    assert np.array_equal(got[short], exp[short])
    # A^T y through the CSC arrays, as the reference does
    At = Csr.transpose_of(S)
    yv = rng.standard_normal(m)
    got_t, _ = _run(bk, At, yv)
    exp_t = po.spmv(At.rp, At.ri, At.rx, yv)
    np.testing.assert_allclose(got_t, exp_t, rtol=1e-12, atol=1e-12)
    short = _short_rows(At)
    assert np.array_equal(got_t[short], exp_t[short])


def test_row_length_classes_and_huge_rows(bk):
    """Every length class side by side on a banded pattern (so the tiles and
    their windows are used; 3% of the entries fall outside): empty rows, one
    lane (<= 64), a warp (65 .. 2048), and rows over a tile's 2048 entries,
    which are read from global memory; tiles cut by the 512-row and
    2048-entry limits."""
    from sovereign_moe_b200 import _lib
    rng = np.random.default_rng(7)
    lens = rng.choice([0, 1, 2, 7, 8, 9, 31, 63, 64, 65, 100, 511, 2047, 2048], size=1500)
    lens = np.concatenate([lens, [2049, 0, 5000, 3, 12000, 0, 0]])
    A, rng = _matrix(lens, 20000, seed=8, banded=True)
    x = rng.standard_normal(A.n)
    got, plan = _run(bk, A, x)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)
    short = _short_rows(A)
    assert np.array_equal(got[short], exp[short])
    info = plan.info()
    assert info["huge_rows"] == 3 and info["entries"] == A.nnz
    assert info["kernel"] == _lib.PDLP_SPMV_PLAN_TILES
    assert info["entries_in_band"] < info["entries"]        # some gathers from global
    got32, _ = _run(bk, A, x, f32=True, plan=plan)
    np.testing.assert_allclose(got32, exp, rtol=1e-4, atol=1e-3)


def test_banded_matrix_stages_windows_and_equals_oracle_bitwise(bk):
    """A multi-period plan (block-bidiagonal with global coupling rows): its
    tiles stage x windows, the few entries outside a window gather from
    global memory, and every row of at most 64 entries equals the oracle."""
    from sovereign_moe_b200.workloads import blending_plan
    S = blending_plan(seed=3, m=20_000, n=60_000, periods=72).problem.A
    A = Csr.of(S)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(A.n)
    got, plan = _run(bk, A, x)
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    short = _short_rows(A)
    assert np.array_equal(got[short], exp[short])
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)
    info = plan.info()
    assert info["kernel"] == 0                           # the tiles, not the fallback
    assert info["banded_tiles"] >= info["tiles"] - 2     # all but the coupling rows' tiles
    assert info["entries_in_band"] > 0.95 * info["entries"]
    At = Csr.transpose_of(S)
    yv = rng.standard_normal(A.m)
    got_t, plan_t = _run(bk, At, yv)
    exp_t = po.spmv(At.rp, At.ri, At.rx, yv)
    assert np.array_equal(got_t, exp_t)        # every column of A has 5 entries
    assert plan_t.info()["entries_in_band"] > 0.9 * A.nnz


@pytest.mark.parametrize("banded", [True, False])
def test_unsorted_rows_keep_storage_order(bk, banded):
    A, rng = _matrix(np.random.default_rng(9).integers(0, 60, 700), 5000, seed=10, sort=False,
                     banded=banded)
    x = rng.standard_normal(A.n)
    got, plan = _run(bk, A, x)
    assert np.array_equal(got, po.spmv(A.rp, A.ri, A.rx, x))
    if banded:
        assert plan.info()["kernel"] == 0


def test_unbanded_pattern_runs_the_row_block_kernel(bk):
    """Fewer than half the entries in a window: the plan runs the streamed
    row-block kernel, with the same results."""
    from sovereign_moe_b200 import _lib
    A, rng = _matrix(np.random.default_rng(13).choice([2, 9, 40, 300], 3000), 200000, seed=14)
    x = rng.standard_normal(A.n)
    got, plan = _run(bk, A, x)
    assert plan.info()["kernel"] == _lib.PDLP_SPMV_PLAN_STREAMED
    np.testing.assert_allclose(got, po.spmv(A.rp, A.ri, A.rx, x), rtol=1e-12, atol=1e-12)


def test_repeat_runs_are_bitwise_and_follow_new_values(bk):
    import torch
    A, rng = _matrix(np.random.default_rng(11).choice([3, 15, 70, 300], 4000), 9000, seed=12,
                     banded=True)
    x = rng.standard_normal(A.n)
    rp, ri = bk.pointer(A.rp), bk.index(A.ri)
    plan = bk.spmv_plan(rp, ri, A.m, A.n)
    first, _ = _run(bk, A, x, plan=plan)
    second, _ = _run(bk, A, x, plan=plan)
    assert np.array_equal(first, second)
    # the plan holds the pattern, not the values: rescaled values are used
    A2 = Csr(A.m, A.n, A.rp, A.ri, A.rx * 3.0)
    third, _ = _run(bk, A2, x, plan=plan)
    np.testing.assert_allclose(third, po.spmv(A.rp, A.ri, A.rx * 3.0, x), rtol=1e-12, atol=1e-12)
    del rp, ri
    torch.cuda.synchronize()


def test_degenerate_shapes(bk):
    # no rows
    A, _ = _matrix(np.zeros(0, np.int64), 10, seed=1)
    got, plan = _run(bk, A, np.ones(10))
    assert got.shape == (0,) and plan.info()["tiles"] == 0
    # one row, empty rows only, one column
    for lens, n in (([5], 8), ([0, 0, 0], 4), ([1] * 1000, 1)):
        A, rng = _matrix(np.array(lens), n, seed=2)
        x = rng.standard_normal(n)
        got, _ = _run(bk, A, x)
        assert np.array_equal(got, po.spmv(A.rp, A.ri, A.rx, x))


def test_pointers_from_an_odd_offset_and_alignment(bk):
    """CSR arrays whose first row starts at entry 5 (rp[0] = 5): the plan
    reads the caller's values from there, whatever their alignment; values
    or x not on a 16-byte boundary are refused by the tile kernel."""
    import torch
    from sovereign_moe_b200 import _lib
    A, rng = _matrix(np.random.default_rng(21).choice([1, 6, 15, 90], 2500), 6000, seed=22,
                     banded=True)
    off = 5
    rp = torch.as_tensor(A.rp + off, device="cuda")
    ri = torch.as_tensor(np.concatenate([np.zeros(off, np.int32), A.ri]), device="cuda")
    rx = torch.as_tensor(np.concatenate([np.full(off, np.nan), A.rx]), device="cuda")
    x = rng.standard_normal(A.n)
    plan = bk.spmv_plan(rp, ri, A.m, A.n)
    assert plan.info()["kernel"] == _lib.PDLP_SPMV_PLAN_TILES
    del rp, ri                                   # the plan holds its own copy of the pattern
    torch.cuda.synchronize()
    out = torch.full((A.m,), POISON, dtype=torch.float64, device="cuda")
    bk.spmv_planned(plan, rx, bk.to_device(x), out)
    assert plan.status(bk._stream()) == 0
    exp = po.spmv(A.rp, A.ri, A.rx, x)
    np.testing.assert_allclose(out.cpu().numpy(), exp, rtol=1e-12, atol=1e-12)
    short = _short_rows(A)
    assert np.array_equal(out.cpu().numpy()[short], exp[short])
    xs = torch.zeros(A.n + 1, dtype=torch.float64, device="cuda")
    code = bk.lib.pdlp_spmv_plan_run_f64(plan._h, rx.data_ptr(), xs[1:].data_ptr(),
                                         out.data_ptr(), bk._stream())
    assert code == _lib.PDLP_ERR_ARG and "aligned" in bk.lib.pdlp_last_error().decode()


def test_plan_rejects_bad_structure(bk):
    import torch
    from sovereign_moe_b200 import _lib
    st = bk._stream()
    h = ctypes.c_void_p()
    rp = torch.tensor([0, 2, 1], dtype=torch.int64, device="cuda")
    ri = torch.tensor([0, 1], dtype=torch.int32, device="cuda")
    assert bk.lib.pdlp_spmv_plan_create(2, 4, rp.data_ptr(), ri.data_ptr(), st,
                                        ctypes.byref(h)) == _lib.PDLP_ERR_ARG
    rp = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    ri = torch.tensor([0, 4], dtype=torch.int32, device="cuda")
    assert bk.lib.pdlp_spmv_plan_create(2, 4, rp.data_ptr(), ri.data_ptr(), st,
                                        ctypes.byref(h)) == _lib.PDLP_ERR_ARG
    assert "out of range" in bk.lib.pdlp_last_error().decode()
    assert bk.lib.pdlp_spmv_plan_create(-1, 4, None, None, st, ctypes.byref(h)) == _lib.PDLP_ERR_ARG
    assert bk.lib.pdlp_spmv_plan_run_f64(None, None, None, None, st) == _lib.PDLP_ERR_ARG


def _rounded(v, f32):
    """The values as the float32 kernel sees them (the oracle takes float64)."""
    return v.astype(np.float32).astype(np.float64) if f32 else v


@pytest.mark.parametrize("f32", [False, True])
def test_back_to_back_products_keep_stream_order(bk, f32):
    """Products launched back to back, each a programmatic dependent of the
    kernel before it (its CTAs stage the plan's arrays while that kernel
    drains): the chain w = A u, u = A^T w, ... reads the previous product's
    output (read after write) and overwrites the vector the previous product
    read (write after read), with a torch kernel between two of the steps.
    Run with a synchronisation after every step, each step equals the oracle
    on its input; run with none, three times over, the chain ends on the
    same bits."""
    import torch
    from sovereign_moe_b200.workloads import blending_plan
    S = blending_plan(seed=5, m=20_000, n=60_000, periods=72).problem.A
    A, At = Csr.of(S), Csr.transpose_of(S)
    dt = torch.float32 if f32 else torch.float64
    pa = bk.spmv_plan(bk.pointer(A.rp), bk.index(A.ri), A.m, A.n)
    pt = bk.spmv_plan(bk.pointer(At.rp), bk.index(At.ri), At.m, At.n)
    assert pa.info()["kernel"] == 0 and pt.info()["kernel"] == 0
    ax, atx = bk.to_device(A.rx).to(dt), bk.to_device(At.rx).to(dt)
    u0 = bk.to_device(np.random.default_rng(6).standard_normal(A.n)).to(dt)

    def chain(u, w, sync):
        snaps = []
        for step in range(6):
            if step % 2 == 0:
                bk.spmv_planned(pa, ax, u, w)
            else:
                bk.spmv_planned(pt, atx, w, u)
                if step == 1:
                    u.mul_(0.125)                  # exact: a power of two
            if sync:
                torch.cuda.synchronize()
                snaps.append((u.clone(), w.clone()))
        return snaps

    u = u0.clone()
    w = torch.full((A.m,), POISON, dtype=dt, device="cuda")
    snaps = chain(u, w, sync=True)
    assert pa.status(bk._stream()) == 0 and pt.status(bk._stream()) == 0
    prev_u = u0.cpu().numpy().astype(np.float64)
    short = _short_rows(A)
    for step, (su, sw) in enumerate(snaps):
        su, sw = su.cpu().numpy().astype(np.float64), sw.cpu().numpy().astype(np.float64)
        if step % 2 == 0:
            exp = po.spmv(A.rp, A.ri, _rounded(A.rx, f32), prev_u)
            if f32:
                np.testing.assert_allclose(sw, exp, rtol=1e-4, atol=1e-3 * np.abs(exp).max())
            else:
                np.testing.assert_allclose(sw, exp, rtol=1e-12, atol=1e-12)
                assert np.array_equal(sw[short], exp[short])
        else:
            exp = po.spmv(At.rp, At.ri, _rounded(At.rx, f32), sw)
            exp = exp * 0.125 if step == 1 else exp
            if f32:
                np.testing.assert_allclose(su, exp, rtol=1e-4, atol=1e-3 * np.abs(exp).max())
            else:
                assert np.array_equal(su, exp)      # every column of A has 5 entries
            prev_u = su
    want_u, want_w = snaps[-1]
    for _ in range(3):
        u = u0.clone()
        w = torch.full((A.m,), POISON, dtype=dt, device="cuda")
        torch.cuda.synchronize()
        chain(u, w, sync=False)
        torch.cuda.synchronize()
        assert torch.equal(u, want_u) and torch.equal(w, want_w)
    assert pa.status(bk._stream()) == 0 and pt.status(bk._stream()) == 0


def test_product_after_copies_into_its_inputs(bk):
    """A product launched right after asynchronous copies into its own
    inputs (x from pinned host memory, the values from another device
    buffer, no synchronisation in between) reads the copied data: the
    dependency on a copy is a full one, like the one on a kernel."""
    import torch
    A, rng = _matrix(np.random.default_rng(31).choice([2, 6, 15, 40], 5000), 12000, seed=32,
                     banded=True)
    plan = bk.spmv_plan(bk.pointer(A.rp), bk.index(A.ri), A.m, A.n)
    assert plan.info()["kernel"] == 0
    rx_dev = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
    x_dev = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    out = torch.full((A.m,), POISON, dtype=torch.float64, device="cuda")
    rx_src = bk.to_device(A.rx)
    for trial in range(3):
        x = rng.standard_normal(A.n)
        x_host = torch.from_numpy(x).pin_memory()
        torch.cuda.synchronize()
        x_dev.copy_(x_host, non_blocking=True)
        rx_dev.copy_(rx_src * float(trial + 1), non_blocking=True)
        bk.spmv_planned(plan, rx_dev, x_dev, out)
        torch.cuda.synchronize()
        exp = po.spmv(A.rp, A.ri, A.rx * float(trial + 1), x)
        short = _short_rows(A)
        assert np.array_equal(out.cpu().numpy()[short], exp[short])
        np.testing.assert_allclose(out.cpu().numpy(), exp, rtol=1e-12, atol=1e-12)
    assert plan.status(bk._stream()) == 0


@pytest.mark.parametrize("f32", [False, True])
def test_full_size_plan_many_tiles_per_cta(bk, f32):
    """The 200k x 600k blending plan of the SpMV bench: about ten tiles per
    CTA in each product, so every stage of the ring is reused over several
    phases by its consumer group (a stage taken on a stale phase shows up
    as wrong rows or as a wait that runs out).  Both products equal the
    oracle (float64 rows of at most 64 entries bit for bit), and a second
    run gives the same bits."""
    import torch
    from sovereign_moe_b200.workloads import blending_plan
    S = blending_plan(seed=0).problem.A
    assert (S.m, S.n) == (200_000, 600_000)
    rng = np.random.default_rng(17)
    for C, v in ((Csr.of(S), rng.standard_normal(S.n)), (Csr.transpose_of(S),
                                                         rng.standard_normal(S.m))):
        got, plan = _run(bk, C, v, f32=f32)
        info = plan.info()
        assert info["kernel"] == 0 and info["tiles"] >= 8 * info["ctas"]
        exp = po.spmv(C.rp, C.ri, _rounded(C.rx, f32), v)
        if f32:
            np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-3 * np.abs(exp).max())
        else:
            short = _short_rows(C)
            assert np.array_equal(got[short], exp[short])
            np.testing.assert_allclose(got, exp, rtol=1e-12, atol=1e-12)
        again, _ = _run(bk, C, v, f32=f32, plan=plan)
        assert np.array_equal(again, got)
    torch.cuda.synchronize()
