"""CPU oracle for the coupled-channel hot path — TEST INFRASTRUCTURE ONLY.

This package restates, in plain NumPy/SciPy, the algorithm that PyTICC uses for
the path that the CUDA library replaces:

* ``oracle.ldmd``         — LDMD log-derivative propagation
                            (``src/pyticc/propagation/logd.py``)
* ``oracle.contraction``  — PotentialGrid → V(R) contraction and W assembly
                            (``src/pyticc/matrix/interaction/common.py``,
                            ``src/pyticc/propagation/runner.py``,
                            ``src/pyticc/matrix/radial.py``)
* ``oracle.matching``     — BF→SF transform, Riccati–Bessel K/S matching
                            (``src/pyticc/match/{asymptotic,smatrix,bessel}.py``)
* ``oracle.pipeline``     — the windowed radial driver and the full solve
                            (``src/pyticc/propagation/runner.py``,
                            ``src/pyticc/scattering/solver.py``)

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference legs may import it, and only as the checker or the timed CPU baseline.
The product (``pyticc_b200``) never imports it and has no CPU fallback.

Parity pin: every function here is checked against golden vectors produced by
running the unmodified reference (``tests/golden/make_golden.py``) and against the
reference's own known-answer tests (``tests/test_oracle_golden.py``).
Third-party arithmetic on the path: ``scipy.special`` (jv, yv, jvp, yvp, kve),
pinned at scipy 1.17.1 by the reference's ``uv.lock``; the oracle calls the
same routines, and NumPy/LAPACK ``solve`` (numpy 2.4.6 pinned; LU with partial
pivoting, as JAX's ``jnp.linalg.solve``).
"""
