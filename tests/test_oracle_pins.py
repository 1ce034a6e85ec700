"""Pins of the CPU oracle against the reference's own verification data.

The reference has no unit tests; its examples verify the solvers against
analytic / manufactured solutions and expected convergence orders.  These tests
run the same set-ups through the oracle at small sizes and assert the error
levels and orders the examples are built to show (O(nx^-2) for periodic
elasticity and Darcy, second-order Dirichlet multigrid, V-cycle residual
reduction, periodic Biot pressure convergence).
"""
import numpy as np
import pytest

import oracle.api as O
from problems import (elastic_material, make_periodic_elasticity, make_walled_elasticity, make_darcy,
                      make_periodic_biot, periodic_elasticity_exact, periodic_biot_exact)

LAM, MU = elastic_material()


def _el_err(nx, levels=1, nt=None):
    P = make_periodic_elasticity(O)
    s = P(lattice=O.LatticeD2Q8("f64/f64"), **{"lambda": LAM}, mu=MU, nx=nx, ny=nx, nz=0,
          precision="f64/f64", io_rate=1 if levels > 1 else 4 * nx * nx, MG_levels=levels)
    s.run(nt if nt is not None else 4 * nx * nx)
    eta = s.records[-1]["eta"][0]
    sig = s.records[-1]["sigma"][0] * nx
    ee, se = periodic_elasticity_exact(nx, nx, LAM, MU)
    res = [r["f_postcollision"] for r in s.records] if levels > 1 else None
    return np.linalg.norm(eta - ee) / np.linalg.norm(ee), np.linalg.norm(sig - se) / np.linalg.norm(se), res


def test_elasticity_periodic_second_order():
    """``examples/elasticity/periodic.py`` (nt = 4 nx^2): O(nx^-2)."""
    e10, s10, _ = _el_err(10)
    e20, s20, _ = _el_err(20)
    assert 0.10 < e10 < 0.13 and 0.025 < e20 < 0.033
    assert 3.5 < e10 / e20 < 4.5 and 3.5 < s10 / s20 < 4.5


def test_elasticity_multigrid_matches_plain_fixed_point():
    """``examples/elasticity/periodic_MG.py``: 50 V-cycles reach the plain solver's
    discretisation error and reduce the relative residual by >1e3."""
    e_plain, _, _ = _el_err(16)
    e_mg, _, res = _el_err(16, levels=3, nt=30)
    assert abs(e_mg - e_plain) < 1e-3 * e_plain
    assert res[-1] / res[0] < 1e-3


def test_elasticity_dirichlet_multigrid_second_order():
    """``examples/elasticity/dirichlet_MG.py`` with full-way bounce-back walls."""
    errs = []
    for n in (16, 32):
        W = make_walled_elasticity(O, "dirichlet")
        s = W(lattice=O.LatticeD2Q8("f64/f64"), **{"lambda": LAM}, mu=MU, nx=n + 2, ny=n + 2, nz=0,
              precision="f64/f64", io_rate=40, MG_levels=3,
              MG_BCs={"top": True, "bottom": True, "left": True, "right": True})
        s.run(40)
        ee, _ = periodic_elasticity_exact(n + 2, n + 2, LAM, MU, -0.5, 2)
        eta = np.array(s.records[-1]["eta"])[0]
        errs.append(np.linalg.norm((eta - ee)[1:-1, 1:-1]) / np.linalg.norm(ee[1:-1, 1:-1]))
    assert errs[0] < 0.2 and 3.5 < errs[0] / errs[1] < 4.8


@pytest.mark.parametrize("kind,lo,hi", [("periodic", 3.0, 4.7), ("neumann", 2.5, 4.5)])
def test_darcy_decay_convergence(kind, lo, hi):
    """``examples/darcy/periodic.py`` and ``neumann_bb.py``: decaying modes with a
    source, errors in the space-time L2 norm of the example."""
    errs = []
    for n in (10, 20):
        nx = n if kind == "periodic" else n + 2
        D = make_darcy(O, kind)
        nt = n * n
        s = D(lattice=O.LatticeD2Q9("f64/f64"), omega=1.0 / (3 * 0.1 + 0.5), nx=nx, ny=nx, nz=0,
              precision="f64/f64", io_rate=max(1, nt // 100))
        s.run(nt)
        sl = (slice(None), slice(None)) if kind == "periodic" else (slice(1, -1), slice(1, -1))
        num = sum(np.linalg.norm((r["rho"][0] - s.exact(r["timestep"]))[sl]) ** 2 for r in s.records)
        den = sum(np.linalg.norm(s.exact(r["timestep"])[sl]) ** 2 for r in s.records)
        errs.append(np.sqrt(num / den))
    assert lo < errs[0] / errs[1] < hi


def test_biot_periodic_pressure_second_order():
    """``examples/poroelasticity/periodic.py`` closed form (centred coupling)."""
    K = 0.1
    errs = []
    for nx in (16, 32):
        PP = make_periodic_biot(O)
        nt = nx * nx // 4
        s = PP(lattice_elasticity=O.LatticeD2Q8("f64/f64"), lattice_darcy=O.LatticeD2Q9("f64/f64"),
               **{"lambda": LAM}, mu=MU, omega=1 / (3 * K + 0.5), alpha=1.0, nx=nx, ny=nx, nz=0,
               precision="f64/f64", io_rate=nt, elasticity_steps=1, elasticity_MG_levels=1)
        s.run(nt)
        r = s.records[-1]
        _, pe = periodic_biot_exact(nx, nx, LAM, MU, 1.0, K, r["timestep"])
        errs.append(np.linalg.norm(r["pressure"][0] - pe) / np.linalg.norm(pe))
    assert errs[0] < 0.02 and errs[0] / errs[1] > 4.0
