"""CPU oracle of the IBIS hourly per-cell step -- TEST INFRASTRUCTURE ONLY.

A float64 NumPy restatement of the reference's ``timestep_body``
(``python-port/ibis/timestepping/loops.py:234-1284``), the per-step
accumulators and hourly wetland CH4 of ``_run_day_inner._step_body``
(``python-port/ibis/timestepping/loops_gswp3.py:115-320``), vectorised over
cells.  Each function cites the reference lines it restates.

Only the test suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline may import this package, and only as the checker or the timed CPU
baseline.  The product (``ibis_b200``) never imports it: the product path
runs the CUDA kernels and fails loudly when they are missing.

Parity of this restatement is pinned against fixtures produced by running the
reference's own JAX source under a NumPy stand-in for ``jax``/``equinox``
(``tests/golden/make_golden.py``), and against the reference's known-answer
tests (``python-port/tests/test_thermo.py`` and friends).
"""
from .step import step, run_steps, new_acc  # noqa: F401
