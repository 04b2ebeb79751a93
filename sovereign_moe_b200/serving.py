"""Continuous-batching LP server on one GPU.

Requests (LPs) arrive over time.  The server keeps a slot table of
device-resident LPs (``BatchEngine``) and runs a loop:

1. move arrived requests into the admission queue;
2. admit queued requests while a slot is free and the LP fits the HBM
   budget -- the engine refuses an LP that does not fit
   (``PDLP_ERR_OOM``) and it waits in the queue until memory frees up;
3. advance every admitted LP by a chunk of engine steps in one persistent
   launch (their work overlaps on the device: one launch serves all of them);
4. fetch and retire the LPs that finished, recording the time from arrival to
   result.

An LP's iterates, step size, primal weight and restarts stay on the device
from admission to retirement; only a small status block crosses to the host
between chunks.  Each result is the same, bit for bit, as the same LP solved
alone (per-LP reductions run over that LP's own tiles in a fixed order).

The reference serves one synchronous solve per request (``ui/server.py:493-540``
calls ``cli.solve`` per POST); ``serve_one_at_a_time`` reproduces that
discipline on the same engine as the baseline the batched form is measured
against.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .batch import BatchEngine
from .pdlp import PDLPParams, solve_pdlp
from .schedule import IterationModel

__all__ = ["Request", "Server", "serve_one_at_a_time", "latency_summary"]


@dataclass
class Request:
    rid: int
    problem: object
    arrival: float                 # seconds from the start of the stream
    admitted: float = float("nan")
    finished: float = float("nan")
    solution: object = None
    slot: int = -1

    @property
    def latency(self):
        return self.finished - self.arrival


@dataclass
class ServeStats:
    completed: int = 0
    makespan: float = 0.0
    chunks: int = 0
    max_concurrent: int = 0
    refused_for_memory: int = 0
    latencies: list = field(default_factory=list)

    @property
    def solves_per_s(self):
        return self.completed / self.makespan if self.makespan > 0 else 0.0


def latency_summary(lat):
    lat = np.asarray(lat, dtype=np.float64)
    if lat.size == 0:
        return {"p50": float("nan"), "p99": float("nan"), "mean": float("nan")}
    return {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "mean": float(lat.mean()), "max": float(lat.max())}


class Server:
    """Continuous batching over a ``BatchEngine`` slot table."""

    def __init__(self, max_slots=64, params: PDLPParams | None = None, chunk_steps=64,
                 memory_budget=0, **engine_kw):
        # a served request must end: infeasible and unbounded LPs are detected
        self.params = params or PDLPParams(device="gpu", eps_abs=1e-6, eps_rel=1e-6,
                                           detect_infeasibility=True)
        self.engine = BatchEngine(max_slots=max_slots, memory_budget=memory_budget, **engine_kw)
        self.max_slots = int(max_slots)
        self.chunk_steps = int(chunk_steps)
        # chunks this many times longer once every request has arrived and
        # none is queued (nothing to admit between chunks)
        self.idle_chunks = 4
        self.queue: deque = deque()
        self.inflight: dict = {}
        # iteration estimates learned from the requests served so far: the
        # engine gives the LPs expected to run longest more blocks
        self.model = IterationModel()

    def close(self):
        self.engine.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _admit_from_queue(self, now, stats):
        while self.queue and len(self.inflight) < self.max_slots:
            req = self.queue[0]
            try:
                slot = self.engine.admit(req.problem, self.params,
                                         hint=self.model.predict(req.problem))
            except _lib.PDLPError as exc:
                if exc.code == _lib.PDLP_ERR_OOM:
                    stats.refused_for_memory += 1
                    if not self.inflight:
                        raise         # nothing will ever free up: the LP alone does not fit
                    return
                raise
            self.queue.popleft()
            req.slot = slot
            req.admitted = now()
            self.inflight[slot] = req
        stats.max_concurrent = max(stats.max_concurrent, len(self.inflight))

    def _harvest(self, now, stats, done):
        st = self.engine.statuses()
        for slot in list(self.inflight):
            if st[slot] != _lib.PDLP_STATUS_RUNNING:
                req = self.inflight.pop(slot)
                req.solution = self.engine.fetch(slot)
                req.finished = now()
                self.model.observe(req.problem, req.solution.iterations)
                self.engine.retire(slot)
                stats.completed += 1
                stats.latencies.append(req.latency)
                done.append(req)

    def serve(self, stream, realtime=True):
        """Serve ``stream`` = [(arrival_seconds, problem), ...].  With
        ``realtime`` the arrivals follow the wall clock (a request cannot be
        admitted before it arrives); otherwise every request is present at 0.
        Returns ``(requests, stats)``."""
        reqs = [Request(i, p, float(t) if realtime else 0.0)
                for i, (t, p) in enumerate(sorted(stream, key=lambda e: e[0]))]
        pending = deque(reqs)
        done: list = []
        stats = ServeStats()
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0

        while pending or self.queue or self.inflight:
            t = now()
            while pending and pending[0].arrival <= t:
                self.queue.append(pending.popleft())
            self._admit_from_queue(now, stats)
            if self.inflight:
                # with nothing left to admit, longer chunks: fewer host round
                # trips (each chunk ends in a synchronisation and a re-plan)
                idle = not pending and not self.queue
                self.engine.step(self.chunk_steps * (self.idle_chunks if idle else 1))
                stats.chunks += 1
                self._harvest(now, stats, done)
            elif pending:
                wait = pending[0].arrival - now()
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        stats.makespan = now()
        return sorted(done, key=lambda r: r.rid), stats


def serve_one_at_a_time(stream, params: PDLPParams | None = None, realtime=True):
    """The baseline discipline: a FIFO queue, one ``solve_pdlp`` at a time
    (the reference server's behaviour), on the same GPU engine."""
    params = params or PDLPParams(device="gpu", eps_abs=1e-6, eps_rel=1e-6,
                                  detect_infeasibility=True)
    reqs = [Request(i, p, float(t) if realtime else 0.0)
            for i, (t, p) in enumerate(sorted(stream, key=lambda e: e[0]))]
    stats = ServeStats()
    t0 = time.perf_counter()
    for req in reqs:
        wait = req.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        req.admitted = time.perf_counter() - t0
        req.solution = solve_pdlp(req.problem, params)
        req.finished = time.perf_counter() - t0
        stats.completed += 1
        stats.latencies.append(req.latency)
    stats.makespan = time.perf_counter() - t0
    return reqs, stats
