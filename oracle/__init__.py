"""CPU oracle for the FDTD time-stepping hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package, and only as the checker. The product
(``meep_torch_b200``) never imports it and has no CPU fallback.

``oracle.fdtd`` restates, in numpy, the algorithm of meep_torch's
``core/pml.py``, ``core/coeffs.py``, ``core/stepper_tm.py``,
``core/stepper_te.py``, ``core/stepper_3d.py``, ``core/sources.py``,
``core/monitors.py``, ``core/monitors_3d.py`` and ``core/run.py``; every
function cites the reference file:line it follows.

Pinning: ``tests/test_oracle_golden.py`` checks this restatement against the
fixtures in ``tests/golden/`` that ``tests/golden/make_golden.py`` produced by
importing and running the reference itself (FP64 and FP32).
"""
