"""The team planner's iteration estimates (``sovereign_moe_b200.schedule``)."""

from types import SimpleNamespace

from sovereign_moe_b200.schedule import IterationModel


def _lp(m, n):
    return SimpleNamespace(A=SimpleNamespace(m=m, n=n))


def test_classes_are_half_octaves_of_columns_per_row():
    c = IterationModel.shape_class
    assert c(100, 200) == 2 and c(100, 283) == 3 and c(100, 800) == 6
    assert c(1000, 2000) == c(50, 100)            # the row count does not matter
    assert c(0, 10) == 0 and c(10, 0) == 0


def test_median_per_class_and_no_estimate_for_unseen_classes():
    mdl = IterationModel(window=3)
    assert mdl.predict(_lp(100, 200)) == 0.0
    for it in (1000, 3000, 2000):
        mdl.observe(_lp(100, 200), it)
    mdl.observe(_lp(300, 600), 9000)               # same class; the window keeps the last 3
    assert mdl.predict(_lp(500, 1000)) == 3000.0   # median of 3000, 2000, 9000
    assert mdl.predict(_lp(100, 800)) == 0.0
    mdl.observe(_lp(100, 800), 0)                  # no iterations: not an observation
    assert mdl.predict(_lp(100, 800)) == 0.0 and len(mdl) == 3
