"""Parity of the CUDA path (through the drop-in classes and the C ABI) with the
CPU oracle on the same seeded inputs.

Tolerances: relative difference <= 1e-12 in FP64 mode and
<= 1e-5 in FP32 mode, measured as max|gpu - oracle| / max|oracle| over the
compared fields.
"""
import numpy as np
import pytest
import torch

import oracle.api as O
from problems import (elastic_material, make_periodic_elasticity, make_walled_elasticity, make_darcy,
                      make_periodic_biot, make_terzaghi)

pytestmark = pytest.mark.gpu

TOL = {"f64/f64": 1e-12, "f32/f32": 1e-5}
LAM, MU = elastic_material()


@pytest.fixture(scope="module")
def G():
    import xlb_biot_b200.api as api
    assert torch.cuda.is_available()
    return api


def rel(a, b):
    a = (a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)).astype(np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / scale) if scale > 0 else float(np.abs(a).max())


def _el(m, prec, cls, **kw):
    return cls(lattice=m.LatticeD2Q8(prec), **{"lambda": LAM}, mu=MU, nz=0, precision=prec, **kw)


@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
@pytest.mark.parametrize("n", [(16, 16), (37, 22)])
def test_elasticity_plain_steps(G, prec, n):
    """Periodic elasticity (examples/elasticity/periodic.py) from a random state,
    20 plain sweeps; odd sizes exercise partial CTAs and the row pitch."""
    nx, ny = n
    Po, Pg = make_periodic_elasticity(O), make_periodic_elasticity(G)
    Po.init_seed = Pg.init_seed = 3
    so, sg = _el(O, prec, Po, nx=nx, ny=ny), _el(G, prec, Pg, nx=nx, ny=ny)
    fo = so.assign_fields_sharded()
    fg = sg.assign_fields_sharded()
    assert rel(fg, fo) < TOL[prec]
    for t in range(20):
        fo, _ = so.step(fo, t)
        fg, _ = sg.step(fg, t)
    assert rel(fg, fo) < TOL[prec] * 10
    eo, so_ = so.update_macroscopic(fo)
    eg, sgm = sg.update_macroscopic(fg)
    assert rel(eg, eo) < TOL[prec] * 10 and rel(sgm, so_) < TOL[prec] * 10
    assert rel(sg.update_divergence(fg), so.update_divergence(fo)) < TOL[prec] * 10


@pytest.mark.parametrize("kind", ["dirichlet", "neumann"])
@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_elasticity_walled_multigrid(G, kind, prec):
    """dirichlet_MG.py / neumann_MG.py: BC rules on every level, 3-level V-cycles,
    residual norms (fstar slot) and fields compared after 4 cycles."""
    kw = dict(nx=18, ny=18, MG_levels=3, MG_BCs={"top": True, "bottom": True, "left": True, "right": True})
    so = _el(O, prec, make_walled_elasticity(O, kind), **kw)
    sg = _el(G, prec, make_walled_elasticity(G, kind), **kw)
    rng = np.random.default_rng(7)
    f0 = (1e-3 * rng.standard_normal((18, 18, 8))).astype(so.precisionPolicy.compute_dtype)
    fo, fg = f0, f0
    for t in range(4):
        fo, ro = so.step(fo, t)
        fg, rg = sg.step(fg, t)
        assert abs(float(rg) - float(ro)) <= TOL[prec] * 10 * abs(float(ro))
    assert rel(fg, fo) < TOL[prec] * 10


def test_elasticity_halfway_dirichlet_rules(G):
    """ElasticityBounceBack (halfway, with wall displacement) on all four sides:
    exercises the reference's zero-padded scatter with D2Q8 direction 0."""
    def make(m):
        class H(m.LBMElasticity):
            def set_boundary_conditions(self):
                bb = self.boundingBoxIndices
                walls = np.concatenate((bb["left"], bb["right"], bb["top"], bb["bottom"]))
                self.BCs.append(m.ElasticityBounceBack(tuple(walls.T), self.gridInfo, self.precisionPolicy,
                                                       np.array([1e-3, -2e-3])))
        return H
    so = _el(O, "f64/f64", make(O), nx=12, ny=10)
    sg = _el(G, "f64/f64", make(G), nx=12, ny=10)
    rng = np.random.default_rng(1)
    f = rng.standard_normal((12, 10, 8))
    fo, fg = f, f
    for t in range(5):
        fo, _ = so.step(fo, t, external_force=0.01 * np.ones((12, 10, 2)))
        fg, _ = sg.step(fg, t, external_force=0.01 * np.ones((12, 10, 2)))
    assert rel(fg, fo) < 1e-12


@pytest.mark.parametrize("kind", ["periodic", "anti", "eq", "neumann"])
@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_darcy_steps(G, kind, prec):
    """examples/darcy/*.py set-ups, 30 sweeps plus moments and gradient."""
    nx = 24 if kind == "periodic" else 26
    kw = dict(omega=1.0 / (3 * 0.1 + 0.5), nx=nx, ny=nx - 4, nz=0, precision=prec)
    so = make_darcy(O, kind)(lattice=O.LatticeD2Q9(prec), **kw)
    sg = make_darcy(G, kind)(lattice=G.LatticeD2Q9(prec), **kw)
    fo = so.assign_fields_sharded()
    fg = sg.assign_fields_sharded()
    assert rel(fg, fo) < TOL[prec]
    ext = 1e-3 * np.random.default_rng(2).standard_normal((nx, nx - 4, 1))
    for t in range(30):
        fo, _ = so.step(fo, t, external_source=ext if t % 2 else None)
        fg, _ = sg.step(fg, t, external_source=ext if t % 2 else None)
    assert rel(fg, fo) < TOL[prec] * 10
    ro, go = so.update_macroscopic(fo, ext, gradient=True)
    rg, gg = sg.update_macroscopic(fg, ext, gradient=True)
    assert rel(rg, ro) < TOL[prec] * 10 and rel(gg, go) < TOL[prec] * 10
    assert rel(sg.gradient(rg, 0.3), so.gradient(ro, 0.3)) < TOL[prec] * 10


def test_darcy_per_cell_omega(G):
    """Extension: per-cell omega (heterogeneous permeability) against the oracle
    with an omega array; a uniform field reproduces the scalar sweep exactly."""
    nx, ny = 20, 16
    rng = np.random.default_rng(5)
    K = np.exp(rng.standard_normal((nx, ny, 1)))
    om = 1.0 / (3 * K + 0.5)
    so = make_darcy(O, "anti")(lattice=O.LatticeD2Q9("f64/f64"), omega=1.0, nx=nx, ny=ny, nz=0, precision="f64/f64")
    so.omega = om
    sg = make_darcy(G, "anti")(lattice=G.LatticeD2Q9("f64/f64"), omega=1.0, nx=nx, ny=ny, nz=0,
                               precision="f64/f64", omega_field=om)
    fo = so.assign_fields_sharded()
    fg = sg.assign_fields_sharded()
    for t in range(10):
        fo, _ = so.step(fo, t)
        fg, _ = sg.step(fg, t)
    assert rel(fg, fo) < 1e-12
    su = make_darcy(G, "anti")(lattice=G.LatticeD2Q9("f64/f64"), omega=0.8, nx=nx, ny=ny, nz=0,
                               precision="f64/f64", omega_field=np.full((nx, ny, 1), 0.8))
    ss = make_darcy(G, "anti")(lattice=G.LatticeD2Q9("f64/f64"), omega=0.8, nx=nx, ny=ny, nz=0, precision="f64/f64")
    f0 = ss.assign_fields_sharded()
    assert torch.equal(su.step(f0, 0)[0], ss.step(f0, 0)[0])


@pytest.mark.parametrize("levels", [1, 2])
@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_biot_periodic(G, levels, prec):
    """examples/poroelasticity/periodic.py: coupled steps with dynamic force and
    source, N(f) inside every smoothing sweep; all seven step outputs compared."""
    K = 0.1
    kw = dict(**{"lambda": LAM}, mu=MU, omega=1 / (3 * K + 0.5), alpha=1.0, nx=16, ny=16, nz=0, precision=prec,
              elasticity_steps=2, elasticity_MG_levels=levels)
    so = make_periodic_biot(O)(lattice_elasticity=O.LatticeD2Q8(prec), lattice_darcy=O.LatticeD2Q9(prec), **kw)
    sg = make_periodic_biot(G)(lattice_elasticity=G.LatticeD2Q8(prec), lattice_darcy=G.LatticeD2Q9(prec), **kw)
    so_state = so.init_state()
    sg_state = sg.init_state()
    for a, b in zip(sg_state, so_state):
        assert rel(a, b) < TOL[prec]
    eo, do, dto = so_state
    eg, dg, dtg = sg_state
    for t in range(6):
        outo = so.step(eo, do, dto, t)
        outg = sg.step(eg, dg, dtg, t)
        eo, do, dto = outo[0], outo[1], outo[4]
        eg, dg, dtg = outg[0], outg[1], outg[4]
    for a, b in zip(outg, outo):
        assert rel(a, b) < TOL[prec] * 100


def test_terzaghi_corner_patched(G):
    """examples/poroelasticity/Terzaghi.py: corner-patched BC subclasses that
    mutate the boundary mask, MG_BCs left/right, k_smooth=4, 3 levels."""
    kw = dict(**{"lambda": LAM}, mu=MU, omega=1.0 / (3 * 0.7 + 0.5), alpha=1.0, nx=18, ny=4, nz=0,
              precision="f64/f64", elasticity_steps=2, elasticity_MG_levels=3, MG_BCs={"left": True, "right": True},
              MG_n_smoothing=4, epsilon=0.5)
    so = make_terzaghi(O)(lattice_elasticity=O.LatticeD2Q8("f64/f64"), lattice_darcy=O.LatticeD2Q9("f64/f64"), **kw)
    sg = make_terzaghi(G)(lattice_elasticity=G.LatticeD2Q8("f64/f64"), lattice_darcy=G.LatticeD2Q9("f64/f64"), **kw)
    eo, do, dto = so.init_state()
    eg, dg, dtg = sg.init_state()
    for t in range(5):
        outo = so.step(eo, do, dto, t)
        outg = sg.step(eg, dg, dtg, t)
        eo, do, dto = outo[0], outo[1], outo[4]
        eg, dg, dtg = outg[0], outg[1], outg[4]
    for a, b in zip(outg, outo):
        assert rel(a, b) < 1e-11


def test_run_loop_output_hooks(G):
    """``run`` drives the ``output_data`` hook with host arrays of the
    reference's shapes (leading gather axis of 1) and MG residual norms."""
    kw = dict(nx=16, ny=16, io_rate=2, MG_levels=2)
    so = _el(O, "f64/f64", make_periodic_elasticity(O), **kw)
    sg = _el(G, "f64/f64", make_periodic_elasticity(G), **kw)
    so.run(4)
    sg.run(4)
    assert len(so.records) == len(sg.records) == 3
    for a, b in zip(sg.records, so.records):
        assert a["timestep"] == b["timestep"]
        assert a["eta"].shape == b["eta"].shape == (1, 16, 16, 2)
        assert rel(a["eta"], b["eta"]) < 1e-12 and rel(a["sigma"], b["sigma"]) < 1e-12
        assert abs(a["f_postcollision"] - b["f_postcollision"]) <= 1e-12 * abs(b["f_postcollision"])


def test_mg_transfers_and_equilibrium(G):
    """_restrict (2x2 block sums), _prolong (injection) and equilibrium."""
    kw = dict(nx=18, ny=14, MG_levels=2, MG_BCs={"left": True, "right": True, "bottom": True, "top": True})
    so = _el(O, "f64/f64", O.LBMElasticity, **kw)
    sg = _el(G, "f64/f64", G.LBMElasticity, **kw)
    rng = np.random.default_rng(11)
    r = rng.standard_normal((18, 14, 8))
    assert rel(sg._restrict(r), so._restrict(r)) < 1e-14
    c = rng.standard_normal((10, 8, 8))
    assert rel(sg._prolong(torch.as_tensor(c, device="cuda")), so._prolong(c)) == 0.0
    eta, sig = rng.standard_normal((18, 14, 2)), rng.standard_normal((18, 14, 3))
    ext = rng.standard_normal((18, 14, 2))
    assert rel(sg.equilibrium(eta, sig, external_force=ext), so.equilibrium(eta, sig, external_force=ext)) < 1e-13


def test_c_abi_rejects_bad_arguments(G):
    """Error behaviour of the C ABI: negative status and a message, no launch."""
    from xlb_biot_b200 import _lib
    g = _lib.Grid(0, 4, 4, 16)
    s = _lib.DarcySweep()
    st = _lib.lib().xlbb_darcy_sweep(0, g, s, None)
    assert st == -1 and b"bad argument" in _lib.lib().xlbb_last_error()
