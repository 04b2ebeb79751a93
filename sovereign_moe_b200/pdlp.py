"""``solve_pdlp`` -- drop-in for ``sovopt.lp.pdlp.solve_pdlp`` on a B200.

Same call, same parameters, same result object as the reference
(``src/sovopt/lp/pdlp.py:79-132, 238-494``): restarted averaged PDHG with the
Ruiz + Pock-Chambolle preconditioner, adaptive step size every
``stepsize_every`` iterations, primal-weight updates and KKT restarts every
``check_every`` iterations, termination judged on the unscaled problem with
the absolute feasibility cap ``feas_cap``.

Everything from preconditioning to the unscaled solution runs on the GPU in
``libpdlp_b200.so``; this module only moves the model in and the solution
out.  There is no CPU path: ``device="cpu"`` raises ``ValueError`` and a
machine without a usable GPU raises ``RuntimeError("GPU backend unavailable
...")``, the reference's error for a missing GPU backend
(``src/sovopt/core/backend.py:321-324``).
"""

from __future__ import annotations

import ctypes
import sys
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .problem import ObjSense, Solution, Status

__all__ = ["PDLPParams", "PDLPInfo", "solve_pdlp", "problem_desc", "params_struct"]


@dataclass
class PDLPParams:
    """Parameters of the reference (``src/sovopt/lp/pdlp.py:79-116``)."""
    eps_abs: float = 1e-8
    eps_rel: float = 1e-8
    feas_cap: float = 1e-6
    max_iter: int = 200_000
    time_limit: float = 600.0
    check_every: int = 64
    stepsize_every: int = 8
    beta_sufficient: float = 0.2
    beta_necessary: float = 0.8
    beta_artificial: float = 0.36
    primal_weight_smoothing: float = 0.5
    scaling: str = "pdlp"
    device: str = "auto"
    verbose: bool = False
    log_every: int = 2000
    # B200 engine only (not in the reference): arithmetic of the iteration's
    # sparse products, "fp64" (the reference's) or "fp32" (float32 values,
    # directions and row sums; iterates and every check stay float64)
    precision: str = "fp64"
    # B200 engine only: end an infeasible LP with a certified status (INFEASIBLE,
    # or INFEASIBLE_OR_UNBOUNDED for a primal ray) instead of running it to its
    # iteration or time limit; off by default, as the reference has no such test
    detect_infeasibility: bool = False
    eps_infeasible: float = 1e-8
    # B200 engine only: the iterations this LP is expected to need (0 = no
    # estimate), a hint for sizing block teams in a batch; results do not
    # depend on it
    expected_iterations: float = 0.0


@dataclass
class PDLPInfo:
    """Solve statistics (``src/sovopt/lp/pdlp.py:119-132``)."""
    iterations: int = 0
    restarts: int = 0
    rejected_steps: int = 0
    primal_res: float = float("nan")
    dual_res: float = float("nan")
    gap: float = float("nan")
    primal_obj: float = float("nan")
    dual_obj: float = float("nan")
    step_size: float = float("nan")
    primal_weight: float = float("nan")
    device: str = "gpu"
    history: list = field(default_factory=list)
    device_seconds: float = 0.0


def _host(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _on_device(a):
    """True for a torch tensor in CUDA memory."""
    return bool(getattr(a, "is_cuda", False))


def _numpy(a, dtype=np.float64):
    """A host view of ``a`` (copied back from the device when it lives there)."""
    if _on_device(a):
        return a.detach().to("cpu").numpy().astype(dtype, copy=False)
    return np.asarray(a, dtype=dtype)


def _device_desc(prob):
    """A ``pdlp_problem_desc`` over CUDA tensors: ``prob``'s arrays stay on the
    device (converted to the ABI's types there when needed) and the engine
    copies them into the slot's arena on the device."""
    import torch
    A = prob.A
    f64, i32, i64 = torch.float64, torch.int32, torch.int64

    def dev(a, dt):
        t = a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a))
        return t.to(device="cuda", dtype=dt).contiguous()

    arrs = dict(rp=dev(A.rp, i64), ri=dev(A.ri, i32), rx=dev(A.rx, f64),
                cp=dev(A.cp, i64), ci=dev(A.ci, i32), cx=dev(A.cx, f64),
                c=dev(prob.c, f64), row_lb=dev(prob.row_lb, f64), row_ub=dev(prob.row_ub, f64),
                col_lb=dev(prob.col_lb, f64), col_ub=dev(prob.col_ub, f64))
    kind = getattr(prob, "kind", None)
    if kind is not None and np.any(_numpy(kind, np.uint8) != 0):
        arrs["kind"] = dev(kind, torch.uint8)
    d = _lib.ProblemDesc()
    d.m, d.n, d.nnz = int(A.m), int(A.n), int(arrs["ci"].numel())
    for name, a in arrs.items():
        setattr(d, name, a.data_ptr() if a.numel() else None)
    for name in ("rp", "cp"):
        setattr(d, name, arrs[name].data_ptr())
    d.obj_offset = float(prob.obj_offset)
    d.sense = -1 if int(prob.sense) == int(ObjSense.MAXIMISE) else 1
    d.memory = _lib.PDLP_MEM_DEVICE
    torch.cuda.current_stream().synchronize()    # conversions done before the engine's stream reads
    return d, arrs


def problem_desc(prob, flip_free=True):
    """A ``pdlp_problem_desc`` over ``prob``'s arrays: host copies, or, when
    the matrix values are a CUDA tensor, the device arrays themselves
    (``_device_desc``).

    Returns ``(desc, keepalive)``; ``keepalive`` must outlive every call that
    uses ``desc``."""
    A = prob.A
    if _on_device(A.rx):
        return _device_desc(prob)
    arrs = dict(
        rp=_host(A.rp, np.int64), ri=_host(A.ri, np.int32), rx=_host(A.rx, np.float64),
        cp=_host(A.cp, np.int64), ci=_host(A.ci, np.int32), cx=_host(A.cx, np.float64),
        c=_host(prob.c, np.float64), row_lb=_host(prob.row_lb, np.float64),
        row_ub=_host(prob.row_ub, np.float64), col_lb=_host(prob.col_lb, np.float64),
        col_ub=_host(prob.col_ub, np.float64))
    kind = getattr(prob, "kind", None)
    if kind is not None and np.any(np.asarray(kind) != 0):
        arrs["kind"] = _host(kind, np.uint8)
    d = _lib.ProblemDesc()
    d.m, d.n, d.nnz = int(A.m), int(A.n), int(arrs["ci"].shape[0])
    for name, a in arrs.items():
        setattr(d, name, a.ctypes.data if a.size else None)
    for name in ("rp", "cp"):
        setattr(d, name, arrs[name].ctypes.data)
    d.obj_offset = float(prob.obj_offset)
    d.sense = -1 if int(prob.sense) == int(ObjSense.MAXIMISE) else 1
    d.memory = _lib.PDLP_MEM_HOST
    return d, arrs


def params_struct(params: PDLPParams, n: int, time_used: float = 0.0, history_capacity=None,
                  power_start="reference"):
    """The C ``pdlp_params`` for ``params``.  ``power_start="reference"`` passes
    the reference's power-iteration start, ``default_rng(0).standard_normal(n)``
    (``pdlp.py:142-143``); ``None`` lets the device generate one."""
    if params.scaling not in _lib.SCALING:
        raise ValueError(f"unknown scaling method {params.scaling!r}; "
                         f"choose from {sorted(_lib.SCALING)}")
    p = _lib.Params()
    _lib.load().pdlp_params_default(ctypes.byref(p))
    p.eps_abs, p.eps_rel, p.feas_cap = params.eps_abs, params.eps_rel, params.feas_cap
    p.max_iter = int(params.max_iter)
    p.time_limit = float(params.time_limit)
    p.check_every, p.stepsize_every = int(params.check_every), int(params.stepsize_every)
    p.beta_sufficient = params.beta_sufficient
    p.beta_necessary = params.beta_necessary
    p.beta_artificial = params.beta_artificial
    p.primal_weight_smoothing = params.primal_weight_smoothing
    p.scaling = _lib.SCALING[params.scaling]
    prec = getattr(params, "precision", "fp64")
    if prec not in _lib.PRECISION:
        raise ValueError(f"unknown precision {prec!r}; choose from {sorted(_lib.PRECISION)}")
    p.precision = _lib.PRECISION[prec]
    p.detect_infeasibility = 1 if getattr(params, "detect_infeasibility", False) else 0
    p.eps_infeasible = float(getattr(params, "eps_infeasible", 1e-8))
    p.expected_iterations = float(getattr(params, "expected_iterations", 0.0))
    p.time_used = float(time_used)
    if history_capacity is None:
        history_capacity = int(min(params.max_iter // max(params.check_every, 1) + 1, 1 << 20))
    p.history_capacity = int(history_capacity)
    keep = None
    if isinstance(power_start, str) and power_start == "reference":
        keep = np.random.default_rng(0).standard_normal(n)
    elif power_start is not None:
        keep = np.ascontiguousarray(power_start, dtype=np.float64)
    p.power_start = keep.ctypes.data if keep is not None and keep.size else None
    return p, keep


def start_with_problem(desc, p, keep_v0):
    """The power-iteration start vector lives where the problem does (the C
    ABI reads it with the problem's memory kind): for a device-resident
    problem the host vector of ``params_struct`` is copied to the device and
    ``p.power_start`` points there.  Returns what must be kept alive."""
    if desc.memory == _lib.PDLP_MEM_DEVICE and keep_v0 is not None and keep_v0.size:
        import torch
        keep_v0 = torch.as_tensor(keep_v0, device="cuda")
        torch.cuda.current_stream().synchronize()
        p.power_start = keep_v0.data_ptr()
    return keep_v0


def _check_device(device: str):
    if device == "cpu":
        raise ValueError("this PDLP engine runs on the GPU only: use device='gpu' or 'auto'")
    if device not in ("auto", "gpu"):
        raise ValueError("device must be 'cpu' or 'gpu'")


def solve_pdlp(prob, params: PDLPParams | None = None) -> Solution:
    """Solve an LP with restarted average PDHG on the GPU.

    ``prob`` is the reference's ``Problem`` (or this package's), with NumPy
    arrays; an object with the same fields whose arrays are torch CUDA
    tensors (``A.rx`` decides) is solved from device memory, without a copy
    through the host.  The result is on the host either way."""
    params = params or PDLPParams()
    t0 = time.perf_counter()
    _check_device(params.device)
    if getattr(prob, "Q", None) is not None:
        raise ValueError("solve_pdlp solves LPs; the model has a quadratic objective")
    lib = _lib.load()
    desc, keep = problem_desc(prob)
    m, n = int(prob.A.m), int(prob.A.n)
    p, keep_v0 = params_struct(params, n, time_used=time.perf_counter() - t0)
    keep_v0 = start_with_problem(desc, p, keep_v0)
    x = np.empty(n)
    y = np.empty(m)
    d = np.empty(n)
    hist = np.empty(5 * max(int(p.history_capacity), 1))
    res = _lib.Result()
    code = lib.pdlp_solve(ctypes.byref(desc), ctypes.byref(p), None, ctypes.byref(res),
                          x.ctypes.data, y.ctypes.data, d.ctypes.data, hist.ctypes.data,
                          _lib.PDLP_MEM_HOST)
    if code == _lib.PDLP_ERR_CUDA:
        msg = lib.pdlp_last_error().decode()
        raise RuntimeError(f"GPU backend unavailable ({msg})")
    _lib.check(code)
    del keep, keep_v0
    return _to_solution(prob, params, res, x, y, d, hist, time.perf_counter() - t0)


def _result_types(prob, params):
    """The classes of the returned objects.

    A caller that passes the reference's own ``Problem``
    (``sovopt.core.problem``) gets the reference's ``Solution`` and ``Status``
    back, and one that passes the reference's ``PDLPParams``
    (``sovopt.lp.pdlp``) gets its ``PDLPInfo``, so code written against sovopt
    keeps working unchanged (``isinstance`` checks, ``Status`` comparisons).
    Any other caller gets this package's classes, which have the same fields
    and integers.  Returns ``(Solution, Status, PDLPInfo)``; this engine's
    extra ``device_seconds`` is set on the info as an attribute."""
    sol_cls, st_cls, info_cls = Solution, Status, PDLPInfo
    mod = sys.modules.get(type(prob).__module__)
    if mod is not None and mod is not sys.modules[Solution.__module__]:
        cand_s, cand_st = getattr(mod, "Solution", None), getattr(mod, "Status", None)
        if isinstance(cand_s, type) and isinstance(cand_st, type):
            sol_cls, st_cls = cand_s, cand_st
    pmod = sys.modules.get(type(params).__module__)
    if pmod is not None and pmod is not sys.modules[__name__]:
        cand_i = getattr(pmod, "PDLPInfo", None)
        if isinstance(cand_i, type):
            info_cls = cand_i
    return sol_cls, st_cls, info_cls


def _to_solution(prob, params, res, x, y, d, hist, elapsed):
    Sol, St, Info = _result_types(prob, params)
    status = St(int(res.status))
    obj = float(_numpy(prob.c) @ x) + float(prob.obj_offset)
    h = hist[:5 * int(res.history_len)].reshape(-1, 5)
    history = [(int(r[0]), float(r[1]), float(r[2]), float(r[3]), float(r[4])) for r in h]
    info = Info(iterations=int(res.iterations), restarts=int(res.restarts),
                rejected_steps=int(res.rejected_steps), primal_res=res.primal_res,
                dual_res=res.dual_res, gap=res.gap, primal_obj=res.primal_obj,
                dual_obj=res.dual_obj, step_size=res.step_size,
                primal_weight=res.primal_weight, device="gpu", history=history)
    info.device_seconds = res.device_seconds
    if params.verbose:
        for (k, pu, du, gu, pou) in history:
            if k % params.log_every == 0:
                print(f"  it {k:>7d}  pres {pu:.2e}  dres {du:.2e}  gap {gu:.2e}  obj {pou:.10g}")
    sol = Sol(status=status, x=x, objective=obj, y=y, reduced_costs=d,
              iterations=int(res.iterations), time=elapsed, method="pdlp[gpu]")
    sol.log = history
    sol.dual_bound = obj
    sol.work_units = float(res.iterations)
    sol.info = info
    return sol.drop_objective_if_unsolved()
