"""CPU oracle for the ADMIXTURE Adam-EM hot path. TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import anything from this package, and only as a checker or as the timed CPU
baseline. The product path (``adamixture_b200``) never imports it.

Contents:

* ``em_oracle``: a float64 numpy restatement of the reference GPU path's algorithm
  (``adamixture/model/em_adam_gpu.py``, ``adamixture/src/utils.py``,
  ``adamixture/src/utils_c/cuda/pack2bit.cu``). Each function cites the reference
  file:line it follows.
* ``refmods``: a loader for the reference's own Cython CPU kernels, which
  ``oracle/Makefile`` compiles from the reference sources into ``oracle/_ref/``.
* ``solvers``: float64 restatements of the per-row solvers (BVLS, the SQP active-set QP,
  the simplex and box projections), the BR-QN gradient/Hessian sums, the randomized-SVD
  products and the CV deviance.
* ``mlp``: a float64 restatement of the warm-start network's forward and backward passes.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference's own Python
implementation (imported from the reference tree in the build container) and the
reference's golden fixtures, and ``tests/test_oracle.py`` checks this oracle against
those vectors.
"""
