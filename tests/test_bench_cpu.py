"""Host logic of ``bench.py`` that needs no GPU: the order in which the CPU
baseline samples the batch."""

from types import SimpleNamespace

import bench


def _lps(sizes):
    return [SimpleNamespace(problem=SimpleNamespace(A=SimpleNamespace(nnz=v))) for v in sizes]


def test_sample_order_is_a_permutation_whose_prefixes_span_the_sizes():
    sizes = [17, 3, 250, 99, 8, 41, 1000, 5, 64, 512, 2, 33, 128, 77, 300, 9]
    order = [k.problem.A.nnz for k in bench.sample_order(_lps(sizes))]
    assert sorted(order) == sorted(sizes)
    ranked = sorted(sizes)
    # the first LPs are the median, then the quartiles: small and large alike
    assert order[0] == ranked[0]
    assert order[1] == ranked[8]
    assert set(order[2:4]) == {ranked[4], ranked[12]}
    for k in (4, 8):
        prefix = sorted(order[:k])
        assert prefix[0] <= ranked[len(sizes) // k] and prefix[-1] >= ranked[-len(sizes) // k - 1]


def test_sample_order_of_a_ragged_count():
    order = [k.problem.A.nnz for k in bench.sample_order(_lps(range(10)))]
    assert sorted(order) == list(range(10)) and order[:3] == [0, 8, 4]
