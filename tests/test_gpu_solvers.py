"""Tolerance drivers and mixed precision against the oracle.

* ``LBMElasticity.solve``: graph-captured pseudo-time loop with FP64 residual
  checks, compared with the oracle after the same number of sweeps;
* FP32 multigrid with an FP64 coarsest level against the all-FP64 oracle at
  the FP32 tolerance;
* Biot step with FP32 elasticity (FP64 coarsest level) and FP64 pressure.
"""
import numpy as np
import pytest
import torch

import oracle.api as O
from problems import elastic_material, make_periodic_elasticity, make_walled_elasticity, make_periodic_biot

pytestmark = pytest.mark.gpu
LAM, MU = elastic_material()


@pytest.fixture(scope="module")
def G():
    import xlb_biot_b200.api as api
    return api


def rel(a, b):
    a = (a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)).astype(np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_plain_solve_to_tolerance_matches_oracle(G):
    kw = dict(**{"lambda": LAM}, mu=MU, nx=16, ny=16, nz=0, precision="f64/f64")
    sg = make_periodic_elasticity(G)(lattice=G.LatticeD2Q8("f64/f64"), **kw)
    f, it, r = sg.solve(tol=1e-6, check_every=50)
    assert r < 1e-6 and it % 2 == 1            # 1 first sweep + even graph batches
    so = make_periodic_elasticity(O)(lattice=O.LatticeD2Q8("f64/f64"), **kw)
    fo = so.assign_fields_sharded()
    for t in range(it):
        fo, _ = so.step(fo, t)
    assert rel(f, fo) < 1e-11


def test_multigrid_solve_with_fp64_coarsest_level(G):
    kw = dict(**{"lambda": LAM}, mu=MU, nx=34, ny=34, nz=0, MG_levels=3,
              MG_BCs={"top": True, "bottom": True, "left": True, "right": True})
    sg = make_walled_elasticity(G, "dirichlet")(lattice=G.LatticeD2Q8("f32/f32"), precision="f32/f32",
                                                coarsest_precision="f64", **kw)
    assert sg._layouts[-1].dtype == torch.float64 and sg._layouts[0].dtype == torch.float32
    so = make_walled_elasticity(O, "dirichlet")(lattice=O.LatticeD2Q8("f64/f64"), precision="f64/f64", **kw)
    rng = np.random.default_rng(3)
    f0 = 1e-3 * rng.standard_normal((34, 34, 8))
    fg, fo = f0, f0
    for t in range(3):
        fg, rg = sg.step(fg, t)
        fo, ro = so.step(fo, t)
    assert rel(fg, fo) < 1e-5
    assert abs(float(rg) - float(ro)) < 1e-4 * abs(float(ro))
    # FP32 residuals bottom out near 1e-5 of the initial one (rounding floor)
    f, it, r = sg.solve(f=fg, tol=1e-4, max_sweeps=60)
    assert r < 1e-4


def test_biot_mixed_precision(G):
    K = 0.1
    kw = dict(**{"lambda": LAM}, mu=MU, omega=1 / (3 * K + 0.5), alpha=1.0, nx=16, ny=16, nz=0,
              elasticity_steps=2, elasticity_MG_levels=2)
    sg = make_periodic_biot(G)(lattice_elasticity=G.LatticeD2Q8("f32/f32"), lattice_darcy=G.LatticeD2Q9("f64/f64"),
                               precision="f32/f32", darcy_precision="f64/f64", coarsest_precision="f64", **kw)
    so = make_periodic_biot(O)(lattice_elasticity=O.LatticeD2Q8("f64/f64"), lattice_darcy=O.LatticeD2Q9("f64/f64"),
                               precision="f64/f64", **kw)
    assert sg.darcy._dtype == torch.float64 and sg.elasticity._dtype == torch.float32
    eg, dg, tg = sg.init_state()
    eo, do, to = so.init_state()
    for t in range(4):
        og = sg.step(eg, dg, tg, t)
        oo = so.step(eo, do, to, t)
        eg, dg, tg = og[0], og[1], og[4]
        eo, do, to = oo[0], oo[1], oo[4]
    assert rel(og[0], oo[0]) < 1e-5          # elasticity populations (FP32)
    assert rel(og[5], oo[5]) < 1e-5          # pressure


@pytest.mark.parametrize("prec,dprec,coarse", [("f64/f64", None, None), ("f32/f32", "f64/f64", "f64")])
def test_biot_step_graph_matches_eager_steps(G, prec, dprec, coarse):
    """The coupled step captured as one CUDA graph replays exactly the eager
    step's kernels: all seven outputs bit-identical after several steps, and
    ``run`` gives the same populations with and without the graph."""
    from xlb_biot_b200.workloads import periodic_biot_1024
    sim = periodic_biot_1024(G, n=64, levels=3, precision=prec, darcy_precision=dprec, coarsest_precision=coarse,
                             max_cycles=2)
    assert sim.graph_capturable()
    graph = sim.capture_step(*sim.init_state())
    graph.load(*sim.init_state())
    e, d, t = sim.init_state()
    for step in range(4):
        eager = sim.step(e, d, t, step)
        e, d, t = eager[0], eager[1], eager[4]
        got = graph.replay()
    for k, (a, b) in enumerate(zip(got, eager)):
        assert torch.equal(a.double(), b.double()), k
    sim.cudaGraph = False
    fe, fd = sim.run(3)
    sim.cudaGraph = True
    ge, gd = sim.run(3)
    assert torch.equal(fe, ge) and torch.equal(fd, gd)


@pytest.mark.parametrize("kind", ["dirichlet", "neumann"])
def test_fp64_arithmetic_residual_sweep_on_fp32_fields(G, kind):
    """``residual_precision="f64"``: the level-0 residual sweep reads FP32
    populations, collides, streams and applies the boundary rules in FP64 and
    rounds only its result.  Near the fixed point (residual << populations) it
    must equal the FP64 sweep of the same (upcast) populations to FP32 rounding
    of the residual itself, which the FP32-arithmetic sweep cannot."""
    kw = dict(**{"lambda": LAM}, mu=MU, nx=34, ny=34, nz=0, MG_levels=2,
              MG_BCs={"top": True, "bottom": True, "left": True, "right": True})
    s64 = make_walled_elasticity(G, kind)(lattice=G.LatticeD2Q8("f64/f64"), precision="f64/f64", **kw)
    s32 = make_walled_elasticity(G, kind)(lattice=G.LatticeD2Q8("f32/f32"), precision="f32/f32",
                                          residual_precision="f64", **kw)
    f, _, _ = s64.solve(tol=1e-9, max_sweeps=300)
    f32 = s32._f(f.float())
    ref = s64._sweep(s64._f(f32.double()), 0, 1.0, -1.0).double().cpu().numpy()
    acc = s32._sweep(f32, 0, 1.0, -1.0, acc64=True).double().cpu().numpy()
    low = s32._sweep(f32, 0, 1.0, -1.0).double().cpu().numpy()
    scale = np.abs(ref).max()
    assert scale > 0
    e_acc = np.abs(acc - ref).max() / scale
    e_low = np.abs(low - ref).max() / scale
    assert e_acc < 1e-5, e_acc
    assert e_low > 100 * e_acc, (e_low, e_acc)     # the test can tell the two apart
