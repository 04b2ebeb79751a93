"""Batched engine: many LPs advanced together by one persistent kernel.

``BatchEngine`` wraps the ``pdlp_batch_*`` entry points of ``libpdlp_b200.so``.
LPs are admitted into slots (their data is copied to the device and
preconditioned there), every ``step`` advances all running slots, and a
finished slot's unscaled solution is fetched and the slot retired.  Each LP
keeps its own step size, primal weight, restart state and termination, and
its per-LP reductions run over its own tiles only, so its result does not
depend on which other LPs share the launch.

The reference has no batched PDLP (its only batched first-order method is the
shared-matrix node relaxation of ``src/sovopt/mip/bnr.py:176-301``); the
per-LP algorithm is exactly ``solve_pdlp``'s.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from .pdlp import (PDLPParams, _check_device, _to_solution, params_struct, problem_desc,
                   start_with_problem)

__all__ = ["BatchEngine"]


class BatchEngine:
    """A slot table of device-resident LPs and the engine that advances them."""

    def __init__(self, max_slots=256, persistent=True, tile_rows=0, tile_nnz=0,
                 lanes_override=0, memory_budget=0, stream=None, barrier_timeout_us=0,
                 autotune=False, test_withhold_arrival=False):
        self.lib = _lib.load()
        cfg = _lib.BatchConfig()
        self.lib.pdlp_batch_config_default(ctypes.byref(cfg))
        cfg.max_slots = int(max_slots)
        cfg.persistent = 1 if persistent else 0
        if tile_rows:
            cfg.tile_rows = int(tile_rows)
        if tile_nnz:
            cfg.tile_nnz = int(tile_nnz)
        cfg.lanes_override = int(lanes_override)
        cfg.memory_budget = int(memory_budget)
        cfg.barrier_timeout_us = int(barrier_timeout_us)
        cfg.autotune = 1 if autotune else 0
        cfg.test_withhold_arrival = 1 if test_withhold_arrival else 0
        h = ctypes.c_void_p()
        code = self.lib.pdlp_batch_create(ctypes.byref(cfg), stream, ctypes.byref(h))
        if code == _lib.PDLP_ERR_CUDA:
            raise RuntimeError(f"GPU backend unavailable ({self.lib.pdlp_last_error().decode()})")
        _lib.check(code)
        self.h = h
        self.max_slots = int(max_slots)
        self._meta = {}

    def close(self):
        if self.h:
            self.lib.pdlp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- slots ------------------------------------------------------------- #

    def admit(self, prob, params: PDLPParams | None = None, power_start="reference", hint=0.0):
        """Copy ``prob`` to the device and precondition it; returns the slot.
        ``hint``: the LP's expected iterations (0 = none), the engine's
        team-sizing hint.  Raises ``PDLPError`` with code ``PDLP_ERR_OOM``
        when it does not fit."""
        params = params or PDLPParams()
        _check_device(params.device)
        t0 = time.perf_counter()
        desc, keep = problem_desc(prob)
        p, keep_v0 = params_struct(params, int(prob.A.n), power_start=power_start)
        keep_v0 = start_with_problem(desc, p, keep_v0)
        if hint:
            p.expected_iterations = float(hint)
        slot = ctypes.c_int32(-1)
        _lib.check(self.lib.pdlp_batch_admit(self.h, ctypes.byref(desc), ctypes.byref(p),
                                             ctypes.byref(slot)))
        del keep, keep_v0
        self._meta[slot.value] = (prob, params, int(p.history_capacity), t0)
        return slot.value

    def admit_many(self, probs, params: PDLPParams | None = None, power_start="reference",
                   hints=None):
        """Admit several LPs with three host synchronisations in all (instead
        of two per LP).  ``hints`` (optional): each LP's expected iterations,
        the engine's team-sizing hint.  Returns ``(slots, codes)``: the slot of
        each LP (-1 when refused) and its return code; a refused LP does not
        stop the others."""
        params = params or PDLPParams()
        _check_device(params.device)
        count = len(probs)
        if count == 0:
            return [], []
        t0 = time.perf_counter()
        descs = (_lib.ProblemDesc * count)()
        prms = (_lib.Params * count)()
        keep = []
        for i, prob in enumerate(probs):
            d, k = problem_desc(prob)
            p, kv = params_struct(params, int(prob.A.n), power_start=power_start)
            kv = start_with_problem(d, p, kv)
            if hints is not None:
                p.expected_iterations = float(hints[i])
            descs[i], prms[i] = d, p
            keep.append((k, kv))
        slots = np.full(count, -1, dtype=np.int32)
        codes = np.zeros(count, dtype=np.int32)
        self.lib.pdlp_batch_admit_many(self.h, count, descs, prms, slots.ctypes.data,
                                       codes.ctypes.data)
        del keep
        for prob, s, p in zip(probs, slots, prms):
            if s >= 0:
                self._meta[int(s)] = (prob, params, int(p.history_capacity), t0)
        return [int(s) for s in slots], [int(c) for c in codes]

    def step(self, max_steps=1 << 16):
        """Advance every running slot; returns how many are still running."""
        active = ctypes.c_int32(0)
        _lib.check(self.lib.pdlp_batch_step(self.h, int(max_steps), ctypes.byref(active)))
        return active.value

    def run(self, chunk=1 << 16):
        """Step until no slot is running."""
        while self.step(chunk) > 0:
            pass

    def poll(self, slot):
        r = _lib.Result()
        _lib.check(self.lib.pdlp_batch_poll(self.h, int(slot), ctypes.byref(r)))
        return r

    def done(self, slot):
        return self.poll(slot).status != _lib.PDLP_STATUS_RUNNING

    def statuses(self):
        """Status of every slot as of the last ``step`` (no device access):
        ``PDLP_STATUS_RUNNING``, a final status, or ``PDLP_SLOT_FREE``."""
        out = np.empty(self.max_slots, dtype=np.int32)
        _lib.check(self.lib.pdlp_batch_statuses(self.h, out.ctypes.data, self.max_slots))
        return out

    def fetch(self, slot):
        """The finished slot's result as a reference ``Solution``."""
        prob, params, hcap, t0 = self._meta[slot]
        r = self.poll(slot)
        m, n = int(prob.A.m), int(prob.A.n)
        x, y, d = np.empty(n), np.empty(m), np.empty(n)
        hist = np.empty(5 * max(hcap, 1))
        _lib.check(self.lib.pdlp_batch_fetch(self.h, int(slot), x.ctypes.data, y.ctypes.data,
                                             d.ctypes.data, hist.ctypes.data, _lib.PDLP_MEM_HOST))
        return _to_solution(prob, params, r, x, y, d, hist, time.perf_counter() - t0)

    def retire(self, slot):
        _lib.check(self.lib.pdlp_batch_retire(self.h, int(slot)))
        self._meta.pop(slot, None)

    def cancel(self, slot):
        _lib.check(self.lib.pdlp_batch_cancel(self.h, int(slot)))

    def scaling(self, slot):
        """The slot's preconditioner: (row factors, column factors, objective
        scale), the reference's ``Scaling.row/col/obj``."""
        prob = self._meta[slot][0]
        r, c = np.empty(int(prob.A.m)), np.empty(int(prob.A.n))
        s = ctypes.c_double()
        _lib.check(self.lib.pdlp_batch_scaling(self.h, int(slot), r.ctypes.data, c.ctypes.data,
                                               ctypes.byref(s), _lib.PDLP_MEM_HOST))
        return r, c, s.value

    def last_timing(self):
        """(device ms, algorithmic PDHG bytes, PDHG iterations) of the last step."""
        ms, by, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        _lib.check(self.lib.pdlp_batch_last_timing(self.h, ctypes.byref(ms), ctypes.byref(by),
                                                   ctypes.byref(it)))
        return ms.value, by.value, it.value

    def slot_bytes(self, m, n, nnz):
        return int(self.lib.pdlp_slot_bytes(int(m), int(n), int(nnz)))

    def solve_all(self, probs, params=None, hints=None):
        """Admit every LP, run to completion, fetch and retire: list of Solutions."""
        slots, codes = self.admit_many(probs, params, hints=hints)
        for c in codes:
            _lib.check(c)
        self.run()
        out = [self.fetch(s) for s in slots]
        for s in slots:
            self.retire(s)
        return out
