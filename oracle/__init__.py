"""CPU oracle for the PDLP path -- TEST INFRASTRUCTURE, not product code.

This package restates, on the CPU, what the reference ``sovopt`` does on its
``--method pdlp`` path, so that the B200 engine can be checked against it on
the same inputs:

* ``oracle.pdlp_oracle``  -- ``solve_pdlp`` and ``scale_problem(method="pdlp")``,
  following ``src/sovopt/lp/pdlp.py`` and ``src/sovopt/numerics/scaling.py``;
* ``oracle.verify_oracle`` -- the independent verifier of ``bench/verify.py``
  with its compensated residual and certified dual bound;
* ``oracle/sparse_ref.c`` -- the sparse kernels, in the reference's own
  accumulation order (built by ``oracle/Makefile``).

Parity is pinned: ``tests/golden/make_golden.py`` ran the reference itself on
a set of LPs and stored its outputs (scale factors, iterates, iteration counts,
objectives, verdicts) under ``tests/golden/``; ``tests/test_oracle_golden.py``
checks this oracle against every one of them.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or the timed CPU
baseline. The product (``sovereign_moe_b200``) never imports it.
"""
