"""Iteration estimates for the engine's team planner.

How many PDHG iterations an LP needs varies by an order of magnitude within
one batch, and the batch's makespan is set by the LPs that need the most.
The engine can give those LPs more blocks when each admitted LP carries an
estimate (``pdlp_params.expected_iterations``).  ``IterationModel``
supplies one: the median iteration count of the LPs already finished in the
same shape class.  The class is the number of columns per row in half
octaves, the shape feature that tracks the iteration count best on the
known-optimum LPs of the batched and served workloads (log iterations against
columns per row correlate at -0.76 on the 256-LP batch; against the row count
at 0.21).  The estimate only moves blocks between LPs: every LP's result is
the same with or without it.
"""

from __future__ import annotations

import math
from collections import defaultdict, deque

import numpy as np

__all__ = ["IterationModel"]


class IterationModel:
    """Median iterations of finished LPs by columns-per-row class."""

    def __init__(self, window: int = 256):
        self.window = int(window)
        self._obs = defaultdict(lambda: deque(maxlen=self.window))

    @staticmethod
    def shape_class(m: int, n: int) -> int:
        if m <= 0 or n <= 0:
            return 0
        return int(round(2.0 * math.log2(n / m)))

    def observe(self, prob, iterations: int):
        """Record a finished LP (its problem and its iteration count)."""
        if iterations > 0:
            self._obs[self.shape_class(prob.A.m, prob.A.n)].append(int(iterations))

    def predict(self, prob) -> float:
        """Expected iterations for ``prob``: the median of its class, or 0
        (no estimate) when no LP of the class has finished yet."""
        seen = self._obs.get(self.shape_class(prob.A.m, prob.A.n))
        return float(np.median(seen)) if seen else 0.0

    def __len__(self):
        return sum(len(v) for v in self._obs.values())
