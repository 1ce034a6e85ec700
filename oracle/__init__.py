"""CPU oracle for the Biot lattice-Boltzmann hot path — TEST INFRASTRUCTURE ONLY.

This package is a plain NumPy restatement of the reference solvers of
s-lunowa/xlb-biot (JAX 0.5.3 code in ``src/elasticity.py``, ``src/darcy.py``,
``src/poroelasticity.py``, ``src/models.py``, ``src/boundary_conditions.py``,
``src/base.py`` and ``src/lattice.py``).  Every function cites the reference ``file:line`` it
follows.  It is used as the checker by ``tests/``, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The
product (``xlb_biot_b200``) never imports it.

Parity status: pinned to the reference's own source.  JAX is not installable
offline, so ``tests/golden/make_golden.py`` runs the unmodified reference
modules under a NumPy stand-in for the JAX array API (``tests/golden/jaxshim``)
and stores their FP64 outputs on seeded cases (``tests/golden/
reference_fixtures.npz``); ``tests/test_golden_reference.py`` holds this
restatement to them at 1e-12 (measured: <= 1e-14).  The analytic and
manufactured solutions of the reference's examples pin it as well
(``tests/test_oracle_pins.py``).

JAX semantics reproduced explicitly (``oracle/jaxsem.py``):
  * ``x.at[idx].set(v)`` with duplicate indices: the last update wins (XLA CPU
    scatter applies updates in index order);
  * ``x.at[idx].add(v)`` with duplicate indices: all updates accumulate;
  * gathers with out-of-range indices clamp, scatters drop them.
"""
