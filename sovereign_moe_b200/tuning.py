"""The engine autotuner: per nnz profile, the lanes that sum each row of the
A and A^T passes and the warp tile shape.

``tune(probs)`` tunes one LP per distinct profile among ``probs``
(``pdlp_tune_lp``: short solo runs of the LP with each candidate, timed on
the device) and leaves the results in the library's process-wide cache;
``BatchEngine(autotune=True)`` (``pdlp_batch_config.autotune``) then applies
them at admission.  ``save``/``load`` keep the cache in a JSON file between
processes.  The reference has no tuner: its kernels use one fixed launch
shape (``src/sovopt/core/backend.py:379-384``).
"""

from __future__ import annotations

import ctypes
import json

from . import _lib
from .pdlp import PDLPParams, params_struct, problem_desc

__all__ = ["profile_key", "tune", "entries", "save", "load", "clear"]

_KEY = ("rows_bucket", "row_len_bucket", "col_len_bucket")
_VAL = ("lanes_rows", "lanes_cols", "tile_rows", "tile_nnz", "us_per_iteration",
        "default_us_per_iteration")


def profile_key(m, n, nnz):
    """The cache key of an LP of this shape: (log2 rows, half-octave mean row
    length of A, half-octave mean row length of A^T)."""
    k = _lib.TuneKey()
    _lib.load().pdlp_tune_key_of(int(m), int(n), int(nnz), ctypes.byref(k))
    return tuple(getattr(k, f) for f in _KEY)


def tune(probs, params: PDLPParams | None = None, stream=None):
    """Tune the first LP of every profile among ``probs`` that the cache does
    not hold yet; returns ``{key: tuning dict}`` for the profiles tuned."""
    lib = _lib.load()
    params = params or PDLPParams(device="gpu")
    have = {tuple(e["key"]) for e in entries()}
    done = {}
    for prob in probs:
        key = profile_key(prob.A.m, prob.A.n, prob.A.nnz)
        if key in have or key in done:
            continue
        desc, keep = problem_desc(prob)
        p, keep_v0 = params_struct(params, int(prob.A.n), power_start=None, history_capacity=0)
        out = _lib.Tuning()
        _lib.check(lib.pdlp_tune_lp(ctypes.byref(desc), ctypes.byref(p), stream,
                                    ctypes.byref(out)))
        del keep, keep_v0
        done[key] = {f: getattr(out, f) for f in _VAL}
    return done


def entries():
    """The cache as a list of ``{"key": [...], **tuning}`` in key order."""
    lib = _lib.load()
    out = []
    for i in range(lib.pdlp_tune_cache_size()):
        k, t = _lib.TuneKey(), _lib.Tuning()
        _lib.check(lib.pdlp_tune_cache_get(i, ctypes.byref(k), ctypes.byref(t)))
        out.append({"key": [getattr(k, f) for f in _KEY], **{f: getattr(t, f) for f in _VAL}})
    return out


def save(path):
    with open(path, "w") as fh:
        json.dump(entries(), fh, indent=1)


def load(path):
    """Put every entry of a saved file into the cache (checked by the library)."""
    lib = _lib.load()
    with open(path) as fh:
        data = json.load(fh)
    for e in data:
        k = _lib.TuneKey(*[int(v) for v in e["key"]])
        t = _lib.Tuning(*[e[f] for f in _VAL])
        _lib.check(lib.pdlp_tune_cache_put(ctypes.byref(k), ctypes.byref(t)))
    return len(data)


def clear():
    _lib.load().pdlp_tune_cache_clear()
