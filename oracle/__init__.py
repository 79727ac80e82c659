"""ORACLE -- test infrastructure, never product code.

A CPU, FP64 restatement of the reference beamtracer's Vlasov-iteration path, used only as
the checker of the CUDA kernels (by ``tests/``, ``__graft_entry__.smoke()``) and as the CPU
baseline that ``bench.py`` times.  The product package ``beamtracer_b200`` never imports
it.

- `kernels`: the three cunumpy kernels of the path (gather, deposit, trace), in C
  (``bt_oracle.c``), with the reference's positional signatures.
- `field`: the staggered edge field (``solver/fields.py:18-67``).
- `poisson`: the finite-volume Poisson operator, linear and Newton solves
  (``solver/poisson.py``; patchwork's operator restated from its documented form).
- `vlasov`: volumes, compensation, mixing and the iteration loop
  (``solver/vlasov.py``, ``solver/tracer.py:678-705``, ``solver/refinement.py:239-296``).
- `diagnostics`: plane moments (``solver/diagnostics.py:56-135``).

Pinned against golden vectors that ``tests/golden/make_golden.py`` generates by running the
reference's own kernel sources and host code in the build container.
"""
