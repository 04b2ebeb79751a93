"""The C-ABI library loads and exports every entry point the header declares
(no compute: these run without a GPU)."""

import ctypes
import os
import re

import numpy as np
import pytest

from sovereign_moe_b200 import _lib
from sovereign_moe_b200.pdlp import PDLPParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "pdlp_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pdlp_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_surface():
    names = declared_functions()
    assert names, "no declarations parsed"
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_abi_version_and_defaults_match_reference_params():
    lib = _lib.load()
    assert lib.pdlp_abi_version() == 5
    p = _lib.Params()
    lib.pdlp_params_default(ctypes.byref(p))
    ref = PDLPParams()
    for f in ("eps_abs", "eps_rel", "feas_cap", "max_iter", "time_limit", "check_every",
              "stepsize_every", "beta_sufficient", "beta_necessary", "beta_artificial",
              "primal_weight_smoothing"):
        assert getattr(p, f) == getattr(ref, f), f
    assert p.scaling == _lib.SCALING["pdlp"]
    # the fields after the reference's: written by the C default at the same offsets
    assert p.precision == _lib.PRECISION["fp64"]
    assert p.detect_infeasibility == 0 and p.eps_infeasible == 1e-8
    assert p.expected_iterations == 0.0    # no scheduling hint
    assert ref.detect_infeasibility is False and ref.eps_infeasible == 1e-8


def test_struct_layouts_match_the_header():
    # sizes of the C structs on x86-64 (natural alignment)
    assert ctypes.sizeof(_lib.ProblemDesc) == 4 + 4 + 8 + 12 * 8 + 8 + 4 + 4
    # six int32, memory_budget, barrier_timeout_us, autotune, test_withhold_arrival
    assert ctypes.sizeof(_lib.BatchConfig) == 6 * 4 + 8 + 8 + 4 + 4
    assert ctypes.sizeof(_lib.TuneKey) == 12
    assert ctypes.sizeof(_lib.Tuning) == 4 * 4 + 2 * 8
    # ..., history_len (+pad), device_seconds, device_start_ns, device_end_ns
    assert ctypes.sizeof(_lib.Result) == 8 + 3 * 8 + 9 * 8 + 8 + 8 + 2 * 8
    # eps..time_limit, check/stepsize, betas + smoothing, scaling (+pad), power_start,
    # time_used, history_capacity + precision, detect (+pad), eps_infeasible,
    # expected_iterations
    assert ctypes.sizeof(_lib.Params) == 5 * 8 + 8 + 4 * 8 + 8 + 8 + 8 + 8 + 8 + 8 + 8


def test_batch_config_defaults():
    lib = _lib.load()
    c = _lib.BatchConfig()
    lib.pdlp_batch_config_default(ctypes.byref(c))
    assert c.block_threads == 128          # the only block size the engine accepts
    assert c.persistent == 1 and c.max_slots == 1
    assert c.barrier_timeout_us == 0       # 0 = the 4 s default
    assert c.autotune == 0                 # the fixed rules unless asked
    assert c.test_withhold_arrival == 0    # the timeout test hook is off


def test_slot_bytes_grows_with_the_problem():
    lib = _lib.load()
    small = lib.pdlp_slot_bytes(100, 300, 1200)
    big = lib.pdlp_slot_bytes(1000, 3000, 12000)
    assert 0 < small < big
    # about 90 bytes per nonzero plus vectors, like the reference's own estimate
    assert big < 200 * 12000 + 400 * 4000


def test_cpu_device_is_refused():
    from sovereign_moe_b200 import solve_pdlp
    from sovereign_moe_b200.workloads import single_small
    with pytest.raises(ValueError):
        solve_pdlp(single_small(0).problem, PDLPParams(device="cpu"))
    with pytest.raises(ValueError):
        solve_pdlp(single_small(0).problem, PDLPParams(device="tpu"))


def test_bnr_engine_refuses_the_cpu_and_fails_loudly_without_a_gpu():
    """The node-relaxation engine has no CPU path: device='cpu' is refused, and
    without a GPU the library's create call fails with a clear error instead of
    falling back."""
    from types import SimpleNamespace
    from sovereign_moe_b200.bnr import BNRConfig, BNREngine
    from sovereign_moe_b200.workloads import node_relaxation
    prob, _, _ = node_relaxation(m=40, n=60, per_col=4, nodes=2)
    with pytest.raises(ValueError):
        BNREngine(prob, SimpleNamespace(obj=1.0), BNRConfig(device="cpu"))
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError, match="GPU backend unavailable"):
            BNREngine(prob, SimpleNamespace(obj=1.0), BNRConfig(batch=2, device="gpu"))


def test_tuning_cache_api_without_a_gpu(tmp_path):
    """The tuner's cache: profile keys, checked entries, save and load."""
    from sovereign_moe_b200 import tuning
    tuning.clear()
    assert tuning.entries() == []
    k = tuning.profile_key(1000, 4000, 32000)
    # log2(1001) = 9.97; 2 log2(33) = 10.09; 2 log2(9) = 6.34
    assert k == (9, 10, 6)
    assert tuning.profile_key(0, 5, 0) == (0, 0, 0)
    lib = _lib.load()
    key = _lib.TuneKey(*k)
    good = _lib.Tuning(2, 1, 32, 256, 11.5, 12.0)
    assert lib.pdlp_tune_cache_put(ctypes.byref(key), ctypes.byref(good)) == _lib.PDLP_OK
    for bad in (_lib.Tuning(3, 1, 32, 256, 1, 1), _lib.Tuning(1, 1, 65, 256, 1, 1),
                _lib.Tuning(1, 1, 32, 513, 1, 1), _lib.Tuning(0, 1, 32, 256, 1, 1)):
        assert lib.pdlp_tune_cache_put(ctypes.byref(key), ctypes.byref(bad)) == _lib.PDLP_ERR_ARG
    e = tuning.entries()
    assert len(e) == 1 and e[0]["key"] == list(k) and e[0]["lanes_rows"] == 2
    path = tmp_path / "tune.json"
    tuning.save(path)
    tuning.clear()
    assert tuning.entries() == []
    assert tuning.load(path) == 1
    assert tuning.entries() == e
    tuning.clear()


def test_struct_sizes_equal_the_compiled_header(tmp_path):
    """Every struct the header declares has the size ctypes gives it, as the
    host C compiler lays it out."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    structs = {"pdlp_problem_desc": _lib.ProblemDesc, "pdlp_params": _lib.Params,
               "pdlp_result": _lib.Result, "pdlp_batch_config": _lib.BatchConfig,
               "pdlp_tune_key": _lib.TuneKey, "pdlp_tuning": _lib.Tuning,
               "pdlp_crossover_info": _lib.CrossoverInfo,
               "pdlp_simplex_params": _lib.SimplexParamsC,
               "pdlp_simplex_info": _lib.SimplexInfo}
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "pdlp_b200.h"\nint main(void) {\n' +
                   "".join(f'  printf("{k} %zu\\n", sizeof({k}));\n' for k in structs) +
                   "  return 0;\n}\n")
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = dict((k, int(v)) for k, v in (line.split() for line in out.splitlines()))
    assert got == {k: ctypes.sizeof(v) for k, v in structs.items()}
