"""CPU oracle for the Biot lattice-Boltzmann hot path — TEST INFRASTRUCTURE ONLY.

This package is a plain NumPy restatement of the reference solvers of
s-lunowa/xlb-biot (JAX 0.5.3 code in ``src/elasticity.py``, ``src/darcy.py``,
``src/poroelasticity.py``, ``src/models.py``, ``src/boundary_conditions.py``,
``src/base.py`` and ``src/lattice.py``).  Every function cites the reference ``file:line`` it
follows.  It is used as the checker by ``tests/``, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The
product (``xlb_biot_b200``) never imports it.

Parity status: the reference needs JAX, which is not installable offline, so no
output of the reference itself could be produced.  The restatement is pinned by
the reference's own verification data instead: the analytic and manufactured
solutions of ``examples/elasticity/*.py``, ``examples/darcy/*.py`` and
``examples/poroelasticity/periodic.py`` (error levels and convergence orders),
see ``tests/test_oracle_pins.py``.  Bitwise-level parity with the JAX code is
therefore "pinned by analytic fixtures", not by golden vectors of the reference.

JAX semantics reproduced explicitly (``oracle/jaxsem.py``):
  * ``x.at[idx].set(v)`` with duplicate indices: the last update wins (XLA CPU
    scatter applies updates in index order);
  * ``x.at[idx].add(v)`` with duplicate indices: all updates accumulate;
  * gathers with out-of-range indices clamp, scatters drop them.
"""
