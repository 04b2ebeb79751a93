"""B200-native engine for sovopt's ``--method pdlp`` path.

``solve_pdlp(prob, params) -> Solution`` keeps the reference's entry point
(``src/sovopt/lp/pdlp.py:238``) and result object; the solve runs in
hand-written sm_100a CUDA kernels behind the C-ABI library
``libpdlp_b200.so`` (declared in ``include/pdlp_b200.h``).  There is no CPU
fallback: without a usable GPU and the built library the call raises.
"""

from .problem import INF, ObjSense, Problem, Solution, SparseMatrix, Status, VarKind

__all__ = ["INF", "ObjSense", "Problem", "Solution", "SparseMatrix", "Status",
           "VarKind", "PDLPParams", "PDLPInfo", "solve_pdlp"]


def __getattr__(name):
    # The solver pulls in torch and the CUDA library; model construction
    # (problem.py, workloads.py) does not need either.
    if name in ("PDLPParams", "PDLPInfo", "solve_pdlp"):
        from . import pdlp
        return getattr(pdlp, name)
    raise AttributeError(name)
