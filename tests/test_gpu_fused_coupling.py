"""The poroelastic smoothing sweep with its coupling force computed in the same
kernel (``xlbb_elast_sweep_divgrad``) against the two-launch form
(``xlbb_elast_divgrad`` then ``xlbb_elast_sweep``): whole coupled Biot steps of
the periodic and the corner-patched Terzaghi set-ups (gradient rules on every
level, FP64 coarsest level under FP32 included) agree bit for bit."""
import numpy as np
import pytest
import torch

from problems import elastic_material, make_periodic_biot, make_terzaghi

pytestmark = pytest.mark.gpu

LAM, MU = elastic_material()


def _run(G, make, fused, prec, steps, **kw):
    sim = make(G)(lattice_elasticity=G.LatticeD2Q8(prec), lattice_darcy=G.LatticeD2Q9(prec), precision=prec,
                  fused_coupling=fused, print_info_rate=0, **kw)
    e, d, dt = sim.init_state()
    for t in range(steps):
        out = sim.step(e, d, dt, t)
        e, d, dt = out[0], out[1], out[4]
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
@pytest.mark.parametrize("levels", [1, 3])
def test_periodic_biot_fused_equals_two_launches(prec, levels):
    import xlb_biot_b200.api as G
    kw = dict(**{"lambda": LAM}, mu=MU, omega=1 / (3 * 0.1 + 0.5), alpha=1.0, nx=32, ny=32, nz=0,
              elasticity_steps=2, elasticity_MG_levels=levels)
    a = _run(G, make_periodic_biot, True, prec, 4, **kw)
    b = _run(G, make_periodic_biot, False, prec, 4, **kw)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_terzaghi_fused_equals_two_launches():
    import xlb_biot_b200.api as G
    kw = dict(**{"lambda": LAM}, mu=MU, omega=1.0 / (3 * 0.7 + 0.5), alpha=1.0, nx=34, ny=8, nz=0,
              elasticity_steps=2, elasticity_MG_levels=3, MG_BCs={"left": True, "right": True}, MG_n_smoothing=4,
              epsilon=0.5, coarsest_precision="f64")
    a = _run(G, lambda m: make_terzaghi(m, ny=8), True, "f32/f32", 4, **kw)
    b = _run(G, lambda m: make_terzaghi(m, ny=8), False, "f32/f32", 4, **kw)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
