"""Benchmark: LP solves/s at rel KKT 1e-6 on the batched B200 PDLP engine.

Workload ("uneven_batch_256"): 256 synthetic LPs of uneven size, rows
log-uniform in 50-5000, columns 2-8x rows, 4-12 nonzeros per column, N(0,1)
values, each built around a known optimum (sovereign_moe_b200.workloads).
One step solves the whole batch to the reference's termination test at
eps_abs = eps_rel = 1e-6 (feas_cap 1e-6, unscaled problem) in one persistent
launch sequence.  The metric is quoted on this batched configuration because
it is a throughput of solves; the single large LP of the blending-plan
configuration does not reach that tolerance within the reference's default
iteration budget, so it serves the per-kernel roofline instead.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value   : solves/s with the LPs already resident in HBM (admission from device
          memory, preconditioning, solve, unscaled solution written to device
          memory), whole job over all ranks.
e2e     : the same through the C ABI from pinned host buffers: H2D of every
          LP's arrays, solve, D2H of x, y and reduced costs, inside the timing.
roofline: the persistent engine kernel; algorithmic bytes of the PDHG
          iterations it ran (24 nnz + 4(m+1) + 4(n+1) + 8(10m + 11n) per
          iteration of an LP, float64) over its CUDA-event time.
--impl reference: the CPU restatement of the reference path (oracle/, same
          iterates as sovopt's solve_pdlp bit for bit) on a bounded sample of
          the same LPs, all host threads, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "uneven_batch_256"
METRIC = "LP solves/s at rel KKT 1e-6"
N_LP = 256
EPS = 1e-6
# DRAM bytes per algorithmic byte of engine_persistent on this batch, from one
# ncu capture of the first 256-step launch of
# `bench.py --workload engine-steps --iters 300`: dram__bytes_read.sum +
# dram__bytes_write.sum = 80.43 GB against 75.90 GB of algorithmic bytes.
TRAFFIC_PER_ALGORITHMIC_BYTE = 80.43 / 75.90


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_batch(seed):
    from sovereign_moe_b200.workloads import uneven_batch
    return uneven_batch(seed=seed, count=N_LP)


def params():
    from sovereign_moe_b200.pdlp import PDLPParams
    return PDLPParams(device="gpu", eps_abs=EPS, eps_rel=EPS)


# --------------------------------------------------------------------------- #
# clocks                                                                       #
# --------------------------------------------------------------------------- #

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during timing."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        busy = [s for s in sm if smax and s > 0.3 * max(smax)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# --------------------------------------------------------------------------- #
# reference arm / CPU baseline                                                 #
# --------------------------------------------------------------------------- #

def sample_order(lps):
    """The batch's LPs in an order whose every prefix spans its size range:
    ranked by nnz, then taken in bit-reversed rank order (the middle, the two
    quartiles, the octiles, ...).  A CPU sample cut off after its first few
    LPs then covers small and large LPs alike instead of the first few of
    the draw."""
    n = len(lps)
    ranked = sorted(range(n), key=lambda i: lps[i].problem.A.nnz)
    bits = max(1, (n - 1).bit_length())
    rev = sorted(range(1 << bits), key=lambda r: int(format(r, f"0{bits}b")[::-1], 2))
    return [lps[ranked[r]] for r in rev if r < n]


def cpu_sample(lps, budget_s):
    """Solve LPs with the CPU oracle, in ``sample_order``, until ``budget_s``
    is spent."""
    from oracle import pdlp_oracle as po
    t0 = time.perf_counter()
    solved = 0
    for k in sample_order(lps):
        s = po.solve_pdlp(k.problem, dict(eps_abs=EPS, eps_rel=EPS))
        if s.status != po.OPTIMAL:
            raise RuntimeError(f"oracle did not converge on {k.problem.name}")
        solved += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return solved, dt, po.num_threads()


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    lps = make_batch(seed=1000)
    budget = args.cpu_budget
    for _ in range(args.warmup and 1):
        cpu_sample(lps[:1], 0.0)                      # C kernels loaded, caches warm
    rates, sample_info = [], None
    for _ in range(args.steps):
        solved, dt, cores = cpu_sample(lps, budget)
        rates.append(solved / dt)
        sample_info = (solved, dt, cores)
    value = statistics.median(rates)
    solved, dt, cores = sample_info
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * N_LP / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lps_per_step": N_LP, "tolerance": "rel KKT 1e-6",
                   "sample": f"{solved} of {N_LP} LPs per step, spread over the size range "
                             f"(bit-reversed nnz rank), {dt:.1f} s"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"{solved} LPs of the {N_LP}-LP batch, spread over its size "
                                   f"range, in {dt:.1f} s"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- #
# GPU arm                                                                      #
# --------------------------------------------------------------------------- #

def device_problem(prob, torch):
    """Device-resident copies of one LP's arrays and a desc over them."""
    from sovereign_moe_b200 import _lib
    from sovereign_moe_b200.problem import ObjSense
    A = prob.A
    t = {
        "rp": torch.as_tensor(A.rp, device="cuda"), "ri": torch.as_tensor(A.ri, device="cuda"),
        "rx": torch.as_tensor(A.rx, device="cuda"), "cp": torch.as_tensor(A.cp, device="cuda"),
        "ci": torch.as_tensor(A.ci, device="cuda"), "cx": torch.as_tensor(A.cx, device="cuda"),
        "c": torch.as_tensor(prob.c, device="cuda"),
        "row_lb": torch.as_tensor(prob.row_lb, device="cuda"),
        "row_ub": torch.as_tensor(prob.row_ub, device="cuda"),
        "col_lb": torch.as_tensor(prob.col_lb, device="cuda"),
        "col_ub": torch.as_tensor(prob.col_ub, device="cuda"),
        "v0": torch.as_tensor(np.random.default_rng(0).standard_normal(A.n), device="cuda"),
    }
    return t, _make_desc(prob, t, _lib.PDLP_MEM_DEVICE)


def host_problem(prob, torch):
    """Pinned host copies of one LP's arrays and a desc over them."""
    from sovereign_moe_b200 import _lib
    A = prob.A
    arrays = {"rp": A.rp, "ri": A.ri, "rx": A.rx, "cp": A.cp, "ci": A.ci, "cx": A.cx,
              "c": prob.c, "row_lb": prob.row_lb, "row_ub": prob.row_ub,
              "col_lb": prob.col_lb, "col_ub": prob.col_ub,
              "v0": np.random.default_rng(0).standard_normal(A.n)}
    t = {k: torch.as_tensor(np.ascontiguousarray(v)).pin_memory() for k, v in arrays.items()}
    return t, _make_desc(prob, t, _lib.PDLP_MEM_HOST)


def _make_desc(prob, t, memory):
    from sovereign_moe_b200 import _lib
    from sovereign_moe_b200.problem import ObjSense
    d = _lib.ProblemDesc()
    d.m, d.n, d.nnz = int(prob.A.m), int(prob.A.n), int(prob.A.nnz)
    for k in ("rp", "ri", "rx", "cp", "ci", "cx", "c", "row_lb", "row_ub", "col_lb", "col_ub"):
        setattr(d, k, t[k].data_ptr())
    d.kind = None
    d.obj_offset = float(prob.obj_offset)
    d.sense = -1 if int(prob.sense) == int(ObjSense.MAXIMISE) else 1
    d.memory = memory
    return d


def h2d_bytes(prob):
    m, n, nnz = prob.A.m, prob.A.n, prob.A.nnz
    return 8 * (m + 1) + 8 * (n + 1) + 2 * 12 * nnz + 8 * (4 * n + 2 * m)


class GpuArm:
    def __init__(self, lps, torch, stream_ptr=None):
        import ctypes
        from sovereign_moe_b200 import _lib
        from sovereign_moe_b200.batch import BatchEngine
        from sovereign_moe_b200.pdlp import params_struct
        self.ctypes = ctypes
        self._lib = _lib
        self.lps = lps
        self.torch = torch
        self.eng = BatchEngine(max_slots=len(lps))
        self.lib = self.eng.lib
        self.p = params()
        self.dev = [device_problem(k.problem, torch) for k in lps]
        self.host = [host_problem(k.problem, torch) for k in lps]
        self.params = []
        for k, (t, _) in zip(lps, self.dev):
            ps, _keep = params_struct(self.p, int(k.problem.A.n), power_start=None,
                                      history_capacity=0)
            ps.power_start = t["v0"].data_ptr()
            self.params.append(ps)
        self.hparams = []
        for k, (t, _) in zip(lps, self.host):
            ps, _keep = params_struct(self.p, int(k.problem.A.n), power_start=None,
                                      history_capacity=0)
            ps.power_start = t["v0"].data_ptr()
            self.hparams.append(ps)
        self.out_dev = [(torch.empty(k.problem.A.n, dtype=torch.float64, device="cuda"),
                         torch.empty(k.problem.A.m, dtype=torch.float64, device="cuda"),
                         torch.empty(k.problem.A.n, dtype=torch.float64, device="cuda"))
                        for k in lps]
        self.out_host = [(torch.empty(k.problem.A.n, dtype=torch.float64).pin_memory(),
                          torch.empty(k.problem.A.m, dtype=torch.float64).pin_memory(),
                          torch.empty(k.problem.A.n, dtype=torch.float64).pin_memory())
                         for k in lps]
        # contiguous descriptor and parameter arrays for pdlp_batch_admit_many
        n = len(lps)
        self.dev_arrays = ((_lib.ProblemDesc * n)(*[d for _, d in self.dev]),
                           (_lib.Params * n)(*self.params))
        self.host_arrays = ((_lib.ProblemDesc * n)(*[d for _, d in self.host]),
                            (_lib.Params * n)(*self.hparams))
        self.single = BatchEngine(max_slots=1)
        # the team planner's iteration estimates, learned from the LPs of the
        # earlier steps (per columns-per-row class; results do not depend on them)
        from sovereign_moe_b200.schedule import IterationModel
        self.model = IterationModel()
        self.latencies = []
        self.engine_ms = 0.0
        self.engine_bytes = 0.0
        self.engine_launches = 0
        self.engine_kernels = 0

    def step(self, host=False):
        """One batched step: admit every LP, run the batch to completion, fetch
        and retire.  Also records each LP's time to tolerance from the start
        of the step: the host's admission time plus the device time from the
        first LP's first engine pass to this LP's end (device clock)."""
        ct, L, c = self.ctypes, self._lib, self.lib
        descs = self.host if host else self.dev
        prms = self.hparams if host else self.params
        outs = self.out_host if host else self.out_dev
        mem = L.PDLP_MEM_HOST if host else L.PDLP_MEM_DEVICE
        darr, parr = (self.host_arrays if host else self.dev_arrays)
        for i, k in enumerate(self.lps):
            parr[i].expected_iterations = self.model.predict(k.problem)
        t0 = time.perf_counter()
        slot_arr = (ct.c_int32 * len(descs))()
        L.check(c.pdlp_batch_admit_many(self.eng.h, len(descs), darr, parr, slot_arr, None))
        slots = list(slot_arr)
        admit_s = time.perf_counter() - t0
        active = ct.c_int32(1)
        while active.value > 0:
            k0 = c.pdlp_launch_count()
            L.check(c.pdlp_batch_step(self.eng.h, 1 << 16, ct.byref(active)))
            self.engine_kernels += c.pdlp_launch_count() - k0
            ms, by, _ = self.eng.last_timing()
            self.engine_ms += ms
            self.engine_bytes += by
            self.engine_launches += 1
        # every LP's result, x, y and d, and the slots retired, with one
        # synchronisation (pdlp_batch_collect_many)
        n = len(slots)
        res = (L.Result * n)()
        ptrs = [(ct.c_void_p * n)(*[o[j].data_ptr() for o in outs]) for j in range(3)]
        L.check(c.pdlp_batch_collect_many(self.eng.h, n, (ct.c_int32 * n)(*slots), res,
                                          ptrs[0], ptrs[1], ptrs[2], None, mem, 1))
        statuses, starts, ends, self.per_lp = [], [], [], []
        for r, k in zip(res, self.lps):
            statuses.append(r.status)
            starts.append(r.device_start_ns)
            ends.append(r.device_end_ns)
            self.model.observe(k.problem, int(r.iterations))
            self.per_lp.append({"m": int(k.problem.A.m), "n": int(k.problem.A.n),
                                "nnz": int(k.problem.A.nnz), "iterations": int(r.iterations),
                                "restarts": int(r.restarts), "start_ns": int(r.device_start_ns),
                                "end_ns": int(r.device_end_ns)})
        first = min(starts)
        self.latencies = [admit_s + (e - first) * 1e-9 for e in ends]
        return statuses

    def one_at_a_time(self, count=None):
        """The plain discipline on the same mix: each LP alone on a one-slot
        engine (admit from pinned host buffers, solve, fetch x/y/d to host,
        retire), one after another.  Returns each LP's service time (s); with
        every LP submitted at the start, LP i's time to tolerance is the sum
        of the service times up to i (first come, first served)."""
        ct, L, c = self.ctypes, self._lib, self.lib
        h = self.single.h
        service = []
        todo = list(zip(self.host, self.hparams, self.out_host))[:count]
        for (t, d), p, (x, y, dd) in todo:
            t0 = time.perf_counter()
            s = ct.c_int32(-1)
            L.check(c.pdlp_batch_admit(h, ct.byref(d), ct.byref(p), ct.byref(s)))
            active = ct.c_int32(1)
            while active.value > 0:
                L.check(c.pdlp_batch_step(h, 1 << 16, ct.byref(active)))
            # result, x, y, d to pinned host buffers and the slot retired with
            # one synchronisation, as the batched arm collects
            r = L.Result()
            one = lambda a: (ct.c_void_p * 1)(a.data_ptr())  # noqa: E731
            L.check(c.pdlp_batch_collect_many(h, 1, (ct.c_int32 * 1)(s.value), ct.byref(r),
                                              one(x), one(y), one(dd), None, L.PDLP_MEM_HOST, 1))
            if r.status != 0:
                raise RuntimeError(f"one-at-a-time solve ended with status {r.status}")
            service.append(time.perf_counter() - t0)
        return service

    def public_one_at_a_time(self, count=None):
        """The same mix through the public drop-in call, solve_pdlp(prob,
        params), one LP after another (a fresh solve per call, as the
        reference's server makes one per request).  Returns service times."""
        from sovereign_moe_b200.pdlp import solve_pdlp
        service = []
        for k in self.lps[:count]:
            t0 = time.perf_counter()
            sol = solve_pdlp(k.problem, self.p)
            if int(sol.status) != 0:
                raise RuntimeError(f"solve_pdlp ended with status {sol.status}")
            service.append(time.perf_counter() - t0)
        return service


def verify_batch(arm, lps):
    """Every result of the last device-resident step against its known optimum
    and the independent verifier."""
    from oracle import verify_oracle as vo
    worst = 0.0
    for k, (x, y, d) in zip(lps, arm.out_dev):
        xh = x.cpu().numpy()
        obj = float(k.problem.c @ xh) + k.problem.obj_offset
        rel = abs(obj - k.f_star) / max(1.0, abs(k.f_star))
        worst = max(worst, rel)
        v = vo.verify(k.problem, xh, obj, feas_tol=1e-6)
        if not v.ok or rel > 1e-6:
            raise RuntimeError(f"{k.problem.name}: rel err {rel:.2e}\n{v.report()}")
    return worst


def rank_max(v, world, device="cuda"):
    """The maximum of ``v`` over the ranks (the timing rule for N > 1)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_gpu(args, rank, world):
    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from sovereign_moe_b200 import _lib
    lib = _lib.load()

    lps = make_batch(seed=1000 + rank)
    arm = GpuArm(lps, torch)
    for _ in range(args.warmup):
        st = arm.step(host=False)
    if any(s != 0 for s in st):
        raise RuntimeError(f"warm-up statuses {set(st)}")
    worst = verify_batch(arm, lps)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return rank_max(v, world, "cuda")

    # device-resident timing
    clocks = ClockSampler(local)
    clocks.start()
    arm.engine_ms = arm.engine_bytes = 0.0
    arm.engine_launches = 0
    arm.engine_kernels = 0
    n0 = lib.pdlp_launch_count()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        st = arm.step(host=False)
    ev1.record()
    barrier()
    launches = lib.pdlp_launch_count() - n0
    clk = clocks.stop()
    dev_ms = ev0.elapsed_time(ev1)
    step_ms = max_over_ranks(dev_ms / args.steps)
    value = N_LP * world / (step_ms / 1000.0)
    eng_ms, eng_bytes, eng_launches = arm.engine_ms, arm.engine_bytes, arm.engine_launches
    eng_kernels = arm.engine_kernels

    # end to end through the C ABI from pinned host buffers (one untimed pass
    # first, so both arms are timed warm)
    arm.step(host=True)
    barrier()
    ev0.record()
    for _ in range(args.steps):
        arm.step(host=True)
    ev1.record()
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    e2e = N_LP * world / (e2e_ms / 1000.0)
    h2d = sum(h2d_bytes(k.problem) for k in lps)
    d2h = sum(8 * (2 * k.problem.A.n + k.problem.A.m) for k in lps)
    lat_batched = list(arm.latencies)
    if args.dump_lps and rank == 0:
        with open(args.dump_lps, "w") as fh:
            json.dump(arm.per_lp, fh)

    # The plain discipline on the same mix, the denominator of the batched
    # form's speed-up: one LP at a time on a one-slot engine, host buffers in
    # and out like e2e (one warm pass over a few LPs first), then through the
    # public solve_pdlp call.
    from sovereign_moe_b200.serving import latency_summary
    service_warm = arm.one_at_a_time(count=4)
    barrier()
    ev0.record()
    service = arm.one_at_a_time()
    ev1.record()
    barrier()
    one_ms = max_over_ranks(ev0.elapsed_time(ev1))
    one_rate = N_LP * world / (one_ms / 1000.0)
    public = None
    if not args.no_public:
        arm.public_one_at_a_time(count=2)
        barrier()
        ev0.record()
        pub_service = arm.public_one_at_a_time()
        ev1.record()
        barrier()
        pub_ms = max_over_ranks(ev0.elapsed_time(ev1))
        public = {"value": N_LP * world / (pub_ms / 1000.0), "unit": "solves/s",
                  "ms": pub_ms, "service_s": latency_summary(pub_service),
                  "call": "solve_pdlp(prob, PDLPParams(eps_abs=1e-6, eps_rel=1e-6)) per LP"}
    del service_warm

    peak, peak_kind = load_peaks()
    achieved = eng_bytes / (eng_ms / 1000.0) / 1e9 if eng_ms > 0 else 0.0

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        solved, dt, cores = cpu_sample(lps, args.cpu_budget)
        cpu = {"value": solved / dt, "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": f"{solved} of the {N_LP} LPs, spread over the size range "
                         f"(bit-reversed nnz rank), solved by the CPU restatement in {dt:.1f} s"}

    served = None
    if rank == 0 and world == 1 and not args.no_serving:
        served = serving_sample()

    if rank == 0:
        total_nnz = sum(k.problem.A.nnz for k in lps)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": e2e / one_rate,
            "vs_baseline_basis": ("e2e solves/s of the batched engine over the plain "
                                  "one-LP-at-a-time GPU PDLP on the same 256 LPs (one-slot "
                                  "engine, pinned host buffers in and out, same tolerance)"),
            "latency_s": dict(latency_summary(lat_batched),
                              definition=("time to rel KKT 1e-6 of each LP from the start of "
                                          "the e2e step (admission of all 256 on the host, "
                                          "then the LP's end on the device clock)")),
            "one_at_a_time": {"value": one_rate, "unit": "solves/s", "ms_per_step": one_ms,
                              "latency_s": dict(latency_summary(np.cumsum(service)),
                                                definition=("every LP submitted at the start, "
                                                            "served first come first served")),
                              "service_s": latency_summary(service),
                              "public_solve_pdlp": public},
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "lps_per_step": N_LP,
                       "rows": "log-uniform 50-5000", "cols": "U{2..8} x rows",
                       "nnz_per_col": "4-12", "total_nnz": int(total_nnz),
                       "tolerance": "rel KKT 1e-6 (eps_abs=eps_rel=1e-6, feas_cap=1e-6)",
                       "l2": "inputs larger than L2 (>126 MB of matrix data per step)",
                       "parallelism": f"replicas x{world}", "worst_rel_obj_err": worst,
                       "scheduling": ("block teams sized by expected remaining iterations: "
                                      "median iterations per columns-per-row class, learned "
                                      "from the LPs finished in earlier steps")},
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (TRAFFIC_PER_ALGORITHMIC_BYTE * eng_bytes / eng_kernels
                                     if eng_kernels else None),
                         "traffic_unit": "bytes per launch (ncu ratio x algorithmic bytes)",
                         "algorithmic_bytes_per_launch": (eng_bytes / eng_kernels
                                                          if eng_kernels else None),
                         "kernel": "engine_persistent", "peak_source": peak_kind,
                         "launches": eng_kernels, "kernel_ms_per_step": eng_ms / args.steps},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(launches),
            "serving": served,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    arm.eng.close()
    arm.single.close()
    return 0


# --------------------------------------------------------------------------- #
# auxiliary workloads (one JSON line each; not the headline metric)            #
# --------------------------------------------------------------------------- #

def _sync_events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_blend(args):
    """Single large LP (200k x 600k, 3M nnz, 720-period blending plan,
    log-uniform values; ``--scale`` shrinks it): float64 vs float32-SpMV
    iteration throughput, the engine kernel's achieved bandwidth, and the
    KKT history, run to rel KKT 1e-6 or ``--iters`` iterations."""
    import torch
    from sovereign_moe_b200.batch import BatchEngine
    from sovereign_moe_b200.pdlp import PDLPParams
    from sovereign_moe_b200.workloads import blending_plan
    sc = args.scale
    k = blending_plan(seed=0, m=int(200_000 * sc), n=int(600_000 * sc),
                      periods=max(1, int(720 * sc)), coupling=max(1, int(30 * sc)))
    peak, kind = load_peaks()
    out = {"workload": f"blending_plan_{k.problem.A.m}_x_{k.problem.A.n}", "nnz": int(k.problem.nnz),
           "iterations": args.iters}
    for prec in ("fp64", "fp32"):
        p = PDLPParams(device="gpu", eps_abs=1e-6, eps_rel=1e-6, max_iter=args.iters,
                       precision=prec)
        with BatchEngine(max_slots=1) as eng:
            slot = eng.admit(k.problem, p)
            ms = by = 0.0
            its = 0
            while True:
                a = eng.step(256)
                m_, b_, i_ = eng.last_timing()
                ms += m_
                by += b_
                its += i_
                if a == 0:
                    break
            r = eng.poll(slot)
            sol = eng.fetch(slot)
            h = sol.log
            pick = sorted(set(list(range(0, len(h), max(1, len(h) // 8))) + [len(h) - 1])) if h else []
            out[prec] = {"ms": ms, "iters": int(r.iterations), "status": int(r.status),
                         "kkt_history": [{"k": h[i][0], "primal_res": h[i][1], "dual_res": h[i][2],
                                          "gap": h[i][3], "primal_obj": h[i][4]} for i in pick],
                         "rel_obj_err_vs_known": abs(sol.objective - k.f_star) / max(1.0, abs(k.f_star)),
                         "us_per_iter": 1000.0 * ms / max(1, r.iterations),
                         "achieved_GBps": by / ms / 1e6 if ms else 0.0,
                         "frac_of_measured_hbm": by / ms / 1e6 / peak if ms else 0.0}
    print(json.dumps({"metric": "PDHG iteration bandwidth (single LP)", "config": out,
                      "peak_GBps": peak, "peak_source": kind}), flush=True)
    return 0


def run_powerlaw(args):
    """1M x 3M, 10M nnz power-law LP: float32 PDHG inner solves, float64
    refinement to rel KKT 1e-8; error against the known optimum."""
    from sovereign_moe_b200.pdlp import PDLPParams
    from sovereign_moe_b200.refine import solve_refined
    from sovereign_moe_b200.workloads import power_law
    scale = args.scale
    k = power_law(seed=0, m=int(1_000_000 * scale), n=int(3_000_000 * scale),
                  nnz=int(10_000_000 * scale))
    t = time.perf_counter()
    s = solve_refined(k.problem, PDLPParams(device="gpu", max_iter=args.iters,
                                            time_limit=args.time_limit), target=1e-8)
    dt = time.perf_counter() - t
    rel = abs(s.objective - k.f_star) / max(1.0, abs(k.f_star))
    print(json.dumps({"metric": "time to rel KKT 1e-8 (refined)", "value": dt, "unit": "s",
                      "status": int(s.status), "rel_obj_err_vs_known": rel,
                      "inner_iterations": int(s.iterations), "rounds": s.log,
                      "config": {"workload": f"power_law_{k.problem.m}x{k.problem.n}",
                                 "nnz": int(k.problem.nnz)}}), flush=True)
    return 0


def run_engine_steps(args):
    """A bounded run of the engine kernel on the headline batch (256 LPs of
    uneven size): admit, run ``--iters`` engine steps in launches of at most
    256 steps (the first launch includes scaling and set-up), report each
    launch.  Small and short enough to capture one launch under a profiler."""
    from sovereign_moe_b200.batch import BatchEngine
    lps = make_batch(1000)
    launches = []
    with BatchEngine(max_slots=len(lps)) as eng:
        for k in lps:
            eng.admit(k.problem, params())
        done = 0
        while done < args.iters:
            n = min(256, args.iters - done)
            active = eng.step(n)
            ms, by, its = eng.last_timing()
            launches.append({"steps": n, "active_after": active, "ms": ms,
                             "us_per_step": 1000.0 * ms / n, "iterations": its,
                             "achieved_GBps": by / ms / 1e6 if ms else 0.0})
            done += n
            if active == 0:
                break
    print(json.dumps({"metric": "engine launches (bounded run)", "launches": launches,
                      "config": {"workload": "uneven_batch_256", "lps": len(lps),
                                 "steps": args.iters}}), flush=True)
    return 0


def run_spmv(args):
    """The standalone CSR SpMV kernel (``pdlp_spmv_f64`` / ``_f32``, the
    reference Backend's ``spmv``) on the large single-LP matrices: the
    blending plan (200k x 600k, 3M nnz) and the power-law LP (1M x 3M, 10M
    nnz at --scale 1), y = A x and y = A^T x.  Each call is timed alone with
    CUDA events after an L2 flush: a 256 MB write followed by a 256 MB read,
    so that the cache holds no dirty lines whose write-back would land in the
    timed call.  Every variant of the row-block pass is timed, then the
    autotuner's choice (``pdlp_spmv_tune_*``) on the same matrix.  The planned
    kernel (``pdlp_spmv_plan_*``) is timed the same way, and also as a stream
    of 30 products over copies of the matrix (at least twice L2 together)
    between one pair of events ("planned_stream", per product)."""
    import ctypes
    import torch
    from sovereign_moe_b200 import _lib
    from sovereign_moe_b200.workloads import blending_plan, power_law
    lib = _lib.load()
    peak, kind = load_peaks()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def flush_l2():
        flush.zero_()
        flush.sum(dtype=torch.int64)

    mats = []
    if args.matrix in ("all", "blending"):
        mats.append(("blending_plan_200k_x_600k", blending_plan(seed=0).problem))
    sc = args.scale
    if args.matrix in ("all", "power_law"):
        mats.append((f"power_law_{int(1e6 * sc)}x{int(3e6 * sc)}",
                     power_law(seed=0, m=int(1_000_000 * sc), n=int(3_000_000 * sc),
                               nnz=int(10_000_000 * sc)).problem))
    names = {_lib.PDLP_SPMV_STREAMED: "streamed", _lib.PDLP_SPMV_ROW_GROUPS: "row_groups",
             _lib.PDLP_SPMV_BANDED: "banded"}
    rows = []
    for name, prob in mats:
        A = prob.A
        for side, (ptr, idx, val, r, c) in (("A x", (A.rp, A.ri, A.rx, A.m, A.n)),
                                            ("A^T y", (A.cp, A.ci, A.cx, A.n, A.m))):
            for prec in ("fp64", "fp32"):
                dt = torch.float64 if prec == "fp64" else torch.float32
                es = 8 if prec == "fp64" else 4
                fn = lib.pdlp_spmv_ex_f64 if prec == "fp64" else lib.pdlp_spmv_ex_f32
                tune = lib.pdlp_spmv_tune_f64 if prec == "fp64" else lib.pdlp_spmv_tune_f32
                rp = torch.as_tensor(np.asarray(ptr, np.int64), device="cuda")
                ri = torch.as_tensor(np.asarray(idx, np.int32), device="cuda")
                rx = torch.as_tensor(np.asarray(val), device="cuda").to(dt)
                x = torch.randn(c, dtype=torch.float64, device="cuda").to(dt)
                y = torch.empty(r, dtype=dt, device="cuda")
                nnz = int(idx.shape[0])
                algo = (es + 4) * nnz + 8 * (r + 1) + es * c + es * r

                def timed(variant):
                    call = lambda: _lib.check(fn(variant, int(r), rp.data_ptr(), ri.data_ptr(),  # noqa: E731
                                                 rx.data_ptr(), x.data_ptr(), y.data_ptr(),
                                                 stream.cuda_stream))
                    for _ in range(3):
                        call()
                    times = []
                    for _ in range(args.steps * 10):
                        flush_l2()
                        e0, e1 = _sync_events(torch)
                        e0.record()
                        call()
                        e1.record()
                        e1.synchronize()
                        times.append(e0.elapsed_time(e1))
                    return statistics.median(times)

                per = {names[v]: timed(v) for v in names}
                # the planned kernel: the pattern analysed once, then one
                # persistent launch per product
                plan = ctypes.c_void_p()
                _lib.check(lib.pdlp_spmv_plan_create(int(r), int(c), rp.data_ptr(), ri.data_ptr(),
                                                     stream.cuda_stream, ctypes.byref(plan)))
                pinfo = _lib.SpmvPlanInfo()
                _lib.check(lib.pdlp_spmv_plan_get_info(plan, ctypes.byref(pinfo)))
                prun = lib.pdlp_spmv_plan_run_f64 if prec == "fp64" else lib.pdlp_spmv_plan_run_f32

                def timed_plan():
                    call = lambda: _lib.check(prun(plan, rx.data_ptr(), x.data_ptr(),  # noqa: E731
                                                   y.data_ptr(), stream.cuda_stream))
                    for _ in range(3):
                        call()
                    times = []
                    for _ in range(args.steps * 10):
                        flush_l2()
                        e0, e1 = _sync_events(torch)
                        e0.record()
                        call()
                        e1.record()
                        e1.synchronize()
                        times.append(e0.elapsed_time(e1))
                    return statistics.median(times)

                per["planned"] = timed_plan()

                # a stream of products, as PDHG makes them: copies of the
                # matrix (indices and values, each with its own plan; together
                # at least twice the 126 MB L2) in turn, 30 products between
                # one pair of events, so each product reads its matrix from
                # HBM and the per-call launch floor is paid once
                ncopies = max(3, -(-260_000_000 // algo))
                copies = [(rp, ri, rx, plan)]
                for _ in range(ncopies - 1):
                    rp2, ri2, rx2 = rp.clone(), ri.clone(), rx.clone()
                    pl2 = ctypes.c_void_p()
                    _lib.check(lib.pdlp_spmv_plan_create(int(r), int(c), rp2.data_ptr(),
                                                         ri2.data_ptr(), stream.cuda_stream,
                                                         ctypes.byref(pl2)))
                    copies.append((rp2, ri2, rx2, pl2))
                for q in range(2 * ncopies):
                    _, _, rxq, plq = copies[q % ncopies]
                    _lib.check(prun(plq, rxq.data_ptr(), x.data_ptr(), y.data_ptr(),
                                    stream.cuda_stream))
                stream_ms = []
                for _ in range(max(3, args.steps)):
                    flush_l2()
                    e0, e1 = _sync_events(torch)
                    e0.record()
                    for q in range(30):
                        _, _, rxq, plq = copies[q % ncopies]
                        _lib.check(prun(plq, rxq.data_ptr(), x.data_ptr(), y.data_ptr(),
                                        stream.cuda_stream))
                    e1.record()
                    e1.synchronize()
                    stream_ms.append(e0.elapsed_time(e1) / 30)
                per["planned_stream"] = statistics.median(stream_ms)
                for _, _, _, plq in copies:
                    _lib.check(lib.pdlp_spmv_plan_status(plq, stream.cuda_stream))
                    lib.pdlp_spmv_plan_destroy(plq)
                del copies
                best = ctypes.c_int32(0)
                tms = (ctypes.c_double * 3)()
                _lib.check(tune(int(r), rp.data_ptr(), ri.data_ptr(), rx.data_ptr(), x.data_ptr(),
                                y.data_ptr(), stream.cuda_stream, 10, ctypes.byref(best), tms))
                ms = per[names[best.value]]
                pms = per["planned"]
                rows.append({"matrix": name, "product": side, "dtype": prec, "rows": int(r),
                             "nnz": nnz, "algorithmic_bytes": algo,
                             "ms_per_variant": per, "tuned_variant": names[best.value],
                             "tuner_ms_warm_l2": {"streamed": tms[0], "row_groups": tms[1],
                                                  "banded": tms[2]},
                             "ms": ms, "GBps": algo / ms / 1e6,
                             "frac_of_measured_hbm": algo / ms / 1e6 / peak,
                             "planned": {"ms": pms, "GBps": algo / pms / 1e6,
                                         "frac_of_measured_hbm": algo / pms / 1e6 / peak,
                                         "stream_ms": per["planned_stream"],
                                         "stream_copies": ncopies,
                                         "stream_frac_of_measured_hbm":
                                             algo / per["planned_stream"] / 1e6 / peak,
                                         "plan_seconds": pinfo.seconds, "tiles": pinfo.tiles,
                                         "banded_tiles": pinfo.banded_tiles,
                                         "entries_in_band": pinfo.entries_in_band,
                                         "huge_rows": pinfo.huge_rows}})
                del rp, ri, rx, x, y
    print(json.dumps({"metric": "SpMV HBM GB/s", "unit": "GB/s", "results": rows,
                      "peak_GBps": peak, "peak_source": kind,
                      "l2": "flushed before every call (256 MB write, then 256 MB read)"}),
          flush=True)
    return 0


def bnr_bytes_per_iteration(m, n, nnz, K):
    """Algorithmic HBM bytes of one batched PDHG iteration over K nodes, every
    trial taken: each (rows, K) float64 block read or written once per kernel
    that touches it -- primal step with its sum (reads X, AtY, AtdY, L, U;
    writes X, AtY, dX: 8 n-blocks), A dX (1 n + 1 m), dual step with its
    sums (reads Y, AX, both A dX; writes Y, AX, dY: 7 m), A^T dY (1 m + 1 n)
    -- plus the CSR and CSC matrices once each."""
    return 8 * (10 * n + 9 * m) * K + 12 * nnz + 8 * (m + 1) + 12 * nnz + 8 * (n + 1)


def run_bnr(args):
    """Batched node relaxation (``sovereign_moe_b200.bnr.BNREngine``, the
    reference's ``sovopt.mip.bnr``): 128 nodes of a 20,000 x 30,000 LP (8 nnz
    per column), 60 PDHG iterations and a safe dual bound per node per call.
    Metric: node bounds per second.  ``value``: one call on device-resident
    bound sets and outputs, L2 flushed (256 MB write) before each; ``e2e``:
    the public ``solve_batch`` with pinned host arrays in and bounds, x and y
    back; ``one_at_a_time``: the same 128 nodes as 128 calls of one node (a
    conventional tree's order); ``cpu_baseline``: the oracle restatement of
    the reference's CPU engine on the same batch, timed over a few iterations
    and scaled to 60."""
    import torch
    from types import SimpleNamespace
    from sovereign_moe_b200 import _lib
    from sovereign_moe_b200.bnr import BNRConfig, BNREngine
    from sovereign_moe_b200.workloads import node_relaxation
    peak, kind = load_peaks()
    K, iters = 128, 60
    prob, L, U = node_relaxation(nodes=K)
    m, n, nnz = prob.A.m, prob.A.n, prob.A.nnz
    sc = SimpleNamespace(obj=1.0)
    eng = BNREngine(prob, sc, BNRConfig(batch=K, iters=iters, device="gpu"))
    lib = eng.lib
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    dev = lambda a: torch.as_tensor(a, device="cuda").contiguous()  # noqa: E731
    dL, dU = dev(L), dev(U)
    dbounds = torch.empty(K, dtype=torch.float64, device="cuda")
    dx = torch.empty((n, K), dtype=torch.float64, device="cuda")
    dy = torch.empty((m, K), dtype=torch.float64, device="cuda")
    dinf = torch.empty(K, dtype=torch.uint8, device="cuda")

    def device_call():
        _lib.check(lib.pdlp_bnr_solve_batch(eng.h, K, dL.data_ptr(), dU.data_ptr(), None, None,
                                            iters, 0.3, 0.6, dbounds.data_ptr(), dx.data_ptr(),
                                            dy.data_ptr(), dinf.data_ptr(), _lib.PDLP_MEM_DEVICE))

    def timed(fn, steps):
        out = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = _sync_events(torch)
            torch.cuda.synchronize()
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return out

    for _ in range(max(3, args.warmup)):
        device_call()
    n0 = lib.pdlp_launch_count()
    dev_ms = timed(device_call, args.steps)
    launches = (lib.pdlp_launch_count() - n0) // max(1, args.steps)
    # e2e through the public API, pinned host buffers
    pin = lambda a: torch.as_tensor(a).pin_memory().numpy()  # noqa: E731
    hL, hU = pin(L), pin(U)
    for _ in range(3):
        eng.solve_batch(hL, hU)
    e2e_ms = timed(lambda: eng.solve_batch(hL, hU), args.steps)
    # one node at a time: 128 calls of K = 1
    one = BNREngine(prob, sc, BNRConfig(batch=1, iters=iters, device="gpu"))
    cols = [(np.ascontiguousarray(L[:, k:k + 1]), np.ascontiguousarray(U[:, k:k + 1]))
            for k in range(K)]
    for k in range(3):
        one.solve_batch(*cols[k])
    one_ms = timed(lambda: [one.solve_batch(*c) for c in cols], 1)[0]
    ms = statistics.median(dev_ms)
    it_bytes = bnr_bytes_per_iteration(m, n, nnz, K)
    gbps = it_bytes * iters / ms / 1e6
    line = {"metric": "BNR node bounds/s", "unit": "nodes/s", "value": K / ms * 1e3,
            "ms_per_step": ms, "steps": args.steps, "warmup": max(3, args.warmup),
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"node_relaxation_{m}x{n}", "nnz": int(nnz), "nodes": K,
                       "iterations": iters, "l2": "flushed before every call (256 MB write)"},
            "gpu_launches": int(launches),
            "e2e": {"value": K / statistics.median(e2e_ms) * 1e3, "unit": "nodes/s",
                    "ms_per_step": statistics.median(e2e_ms),
                    "h2d_bytes_per_step": int(L.nbytes + U.nbytes),
                    "d2h_bytes_per_step": int(8 * K + 8 * n * K + 8 * m * K + K)},
            "one_at_a_time": {"value": K / one_ms * 1e3, "unit": "nodes/s", "ms": one_ms},
            "roofline": {"bound": "hbm", "achieved": gbps, "peak": peak, "unit": "GB/s",
                         "frac": gbps / peak, "peak_source": kind,
                         "algorithmic_bytes_per_iteration": it_bytes,
                         "note": "whole call (60 iterations + bound) against the iterations' bytes"}}
    if not args.no_cpu:
        import oracle.bnr_oracle as bo
        A = prob.A
        o = bo.BNROracle(A.rp, A.ri, A.rx, A.cp, A.ci, A.cx, prob.c, prob.row_lb, prob.row_ub,
                         1.0, 0.0, batch=K, iters=4)
        t0 = time.perf_counter()
        o.solve_batch(L, U)
        t = (time.perf_counter() - t0) * iters / 4
        line["cpu_baseline"] = {"value": K / t, "unit": "nodes/s", "cores": 1, "kind": "port",
                                "sample": f"{K} nodes x 4 iterations (+ bound), scaled to {iters}"}
    print(json.dumps(line), flush=True)
    return 0


def run_tune(args):
    """The engine autotuner on the headline batch (256 uneven LPs): tune one
    LP per nnz profile (``sovereign_moe_b200.tuning.tune``), then solve the
    batch with the engine's fixed rules and with the tuned choices, each
    device-resident like the headline ``value`` (3 warm-up batches, then
    ``--steps`` timed ones), and report both rates and the tuning cost."""
    import torch
    from sovereign_moe_b200 import tuning
    from sovereign_moe_b200.batch import BatchEngine
    lps = make_batch(seed=1000)
    probs = [k.problem for k in lps]
    tuning.clear()
    t0 = time.perf_counter()
    done = tuning.tune(probs, params())
    tune_s = time.perf_counter() - t0
    out = {}
    for mode in ("fixed", "tuned"):
        with BatchEngine(max_slots=len(probs), autotune=(mode == "tuned")) as eng:
            for _ in range(3):
                eng.solve_all(probs, params())
            e0, e1 = _sync_events(torch)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(args.steps):
                sols = eng.solve_all(probs, params())
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
        worst = max(abs(s.objective - k.f_star) / max(1.0, abs(k.f_star))
                    for s, k in zip(sols, lps))
        out[mode] = {"solves_per_s": len(probs) / (ms / 1000.0), "ms_per_batch": ms,
                     "worst_rel_obj_err": worst}
    gains = [v["default_us_per_iteration"] / v["us_per_iteration"] for v in done.values()]
    print(json.dumps({"metric": "autotuned engine: LP solves/s at rel KKT 1e-6",
                      "unit": "solves/s", "fixed": out["fixed"], "tuned": out["tuned"],
                      "ratio_tuned_over_fixed": out["tuned"]["solves_per_s"] / out["fixed"]["solves_per_s"],
                      "profiles_tuned": len(done), "tuning_s": tune_s,
                      "solo_gain_per_profile": {"min": min(gains), "median": statistics.median(gains),
                                                "max": max(gains)},
                      "choices": [{"key": list(k), **v} for k, v in done.items()],
                      "config": {"workload": WORKLOAD, "lps": len(probs)}}), flush=True)
    tuning.clear()
    return 0


def run_precision(args):
    """FP32-SpMV against float64 per instance: config-1-shaped known-optimum
    LPs (230 x 2025, seeds 0-7) and 8 LPs of the uneven batch, each solved at
    rel KKT 1e-6 in both modes; objective error against the known optimum and
    between the modes, iterations of each."""
    from sovereign_moe_b200.batch import BatchEngine
    from sovereign_moe_b200.pdlp import PDLPParams
    from sovereign_moe_b200.workloads import single_small, uneven_batch
    cases = [(f"single_small_s{s}", single_small(seed=s)) for s in range(8)]
    cases += [(k.problem.name, k) for k in uneven_batch(seed=1000, count=8)]
    rows = []
    for name, k in cases:
        out = {}
        for prec in ("fp64", "fp32"):
            p = PDLPParams(device="gpu", eps_abs=EPS, eps_rel=EPS, precision=prec)
            with BatchEngine(max_slots=1) as eng:
                out[prec] = eng.solve_all([k.problem], p)[0]
        f = float(k.f_star)
        scale = max(1.0, abs(f))
        rows.append({"lp": name, "rows": int(k.problem.A.m), "cols": int(k.problem.A.n),
                     "status": [int(out["fp64"].status), int(out["fp32"].status)],
                     "iterations": [int(out["fp64"].iterations), int(out["fp32"].iterations)],
                     "rel_err_fp64": abs(out["fp64"].objective - f) / scale,
                     "rel_err_fp32": abs(out["fp32"].objective - f) / scale,
                     "rel_diff_fp32_fp64": abs(out["fp32"].objective - out["fp64"].objective) / scale,
                     "max_abs_dx": float(np.max(np.abs(out["fp32"].x - out["fp64"].x)))})
    print(json.dumps({"metric": "FP32-SpMV vs FP64 per instance", "tolerance": "rel KKT 1e-6",
                      "results": rows}), flush=True)
    return 0


def serving_sample(count=96, rate=1000.0, max_rows=2000, slots=128):
    """Config 5's small class (rows up to 2,000: 70% of the mixture) as a
    Poisson stream of ``count`` requests at ``rate`` per second, served with
    continuous batching (``serving.Server``) and, on the same GPU, one
    ``solve_pdlp`` at a time in arrival order (the reference server's
    discipline); every objective is checked against its known optimum."""
    from sovereign_moe_b200.serving import Server, latency_summary, serve_one_at_a_time
    from sovereign_moe_b200.workloads import serving_stream
    stream = serving_stream(seed=0, count=count, rate=rate, max_rows=max_rows)
    items = [(t, k.problem) for t, k in stream]
    with Server(max_slots=slots) as srv:
        done, st = srv.serve(items)
    one, st1 = serve_one_at_a_time(items)
    wrong = sum(1 for r, (t, k) in zip(done, stream)
                if abs(r.solution.objective - k.f_star) / max(1.0, abs(k.f_star)) > 1e-6)
    return {"value": st.solves_per_s, "unit": "solves/s",
            "latency_s": latency_summary(st.latencies),
            "one_at_a_time": {"value": st1.solves_per_s, "unit": "solves/s",
                              "latency_s": latency_summary(st1.latencies)},
            "speedup_vs_one_at_a_time": st.solves_per_s / max(st1.solves_per_s, 1e-12),
            "max_concurrent": st.max_concurrent, "objectives_off_by_over_1e-6": wrong,
            "config": {"workload": "poisson_small_class", "count": count, "rate_per_s": rate,
                       "max_rows": max_rows, "slots": slots,
                       "timing": "wall clock, host server loop included in both arms"}}


def run_serving(args):
    """Poisson arrivals served with continuous batching vs one at a time."""
    from sovereign_moe_b200.serving import Server, latency_summary, serve_one_at_a_time
    from sovereign_moe_b200.workloads import serving_stream
    stream = serving_stream(seed=0, count=args.count, rate=args.rate, max_rows=args.max_rows)
    items = [(t, k.problem) for t, k in stream]
    with Server(max_slots=args.slots) as srv:
        done, st = srv.serve(items)
    one, st1 = serve_one_at_a_time(items)
    bad = [r.rid for r, (t, k) in zip(done, stream)
           if abs(r.solution.objective - k.f_star) / max(1.0, abs(k.f_star)) > 1e-6]
    print(json.dumps({"metric": "served LP solves/s at rel KKT 1e-6", "value": st.solves_per_s,
                      "unit": "solves/s", "latency_s": latency_summary(st.latencies),
                      "one_at_a_time": {"value": st1.solves_per_s,
                                        "latency_s": latency_summary(st1.latencies)},
                      "speedup_vs_one_at_a_time": st.solves_per_s / max(st1.solves_per_s, 1e-12),
                      "max_concurrent": st.max_concurrent, "wrong": bad,
                      "config": {"workload": "poisson_mixture", "rate_per_s": args.rate,
                                 "count": args.count, "max_rows": args.max_rows}}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0,
                    help="seconds of CPU work per timed CPU sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--dump-lps", default=None,
                    help="write each LP's size, iterations and device start/end (JSON)")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the served-stream sample after the timed steps")
    ap.add_argument("--no-public", action="store_true",
                    help="skip the one-at-a-time pass through the public solve_pdlp")
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "blend", "powerlaw", "serving", "engine-steps", "spmv",
                             "precision", "bnr", "tune"],
                    help="batch: the headline metric; the others print auxiliary lines")
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--matrix", default="all", choices=["all", "blending", "power_law"],
                    help="matrices of --workload spmv")
    ap.add_argument("--time-limit", type=float, default=600.0)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--count", type=int, default=200)
    ap.add_argument("--slots", type=int, default=128)
    ap.add_argument("--max-rows", type=int, default=None)
    args = ap.parse_args()
    if args.workload == "blend":
        return run_blend(args)
    if args.workload == "powerlaw":
        return run_powerlaw(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "engine-steps":
        return run_engine_steps(args)
    if args.workload == "spmv":
        return run_spmv(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "bnr":
        return run_bnr(args)
    if args.workload == "tune":
        return run_tune(args)
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_gpu(args, rank, world)


if __name__ == "__main__":
    sys.exit(main())
