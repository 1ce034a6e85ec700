"""Pipeline 4 (four columns per lane for eligible FP32 elasticity sweeps)
against pipeline 3 (one thread per cell): bit-identical outputs of the damped
smoothing sweep, the plain step, the residual-corrected sweep and a sweep
without external force, on periodic grids spanning several 128-column tiles,
with a short last tile and a row count off the 16-row tile height; sweeps that
do not qualify (fused sums, small grids) stay on the one-thread-per-cell
kernel."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _elasticity(G, nx, ny):
    return G.LBMElasticity(lattice=G.LatticeD2Q8("f32/f32"), **{"lambda": 0.1}, mu=0.08, nx=nx, ny=ny, nz=0,
                           precision="f32/f32", MG_levels=1, print_info_rate=0)


@pytest.mark.parametrize("shape", [(256, 256), (320, 250), (1024, 64), (96, 768)])
def test_four_column_sweep_identical_to_push(shape):
    import xlb_biot_b200.api as G
    from xlb_biot_b200 import autotune
    nx, ny = shape
    el = _elasticity(G, nx, ny)
    L = el._L(0)
    g = torch.Generator(device="cpu").manual_seed(nx + ny)
    f = L.field(torch.randn(nx, ny, 8, generator=g, dtype=torch.float64), 8)
    fe = L.field(torch.randn(nx, ny, 2, generator=g, dtype=torch.float64), 2)
    r = L.field(torch.randn(nx, ny, 8, generator=g, dtype=torch.float64), 8)
    calls = [dict(a=0.25, b=0.75, fext=fe), dict(fext=fe), dict(a=1.0, b=-1.0, resid=r, fext=fe),
             dict(a=0.25, b=0.75)]
    saved = autotune.get_config(autotune.ELASTICITY)
    outs = []
    try:
        for pipe in (3, 4):
            autotune.set_config(autotune.ELASTICITY, 128, 1, 1, 8, pipe)
            assert [el._sweep(f, 0, query=True, **kw) for kw in calls] == [pipe] * len(calls)
            outs.append([el._sweep(f, 0, **kw) for kw in calls])
    finally:
        autotune.set_config(autotune.ELASTICITY, **saved)
    for i, (x, y) in enumerate(zip(*outs)):
        assert torch.equal(x, y), (shape, calls[i].keys())


def test_four_column_sweep_eligibility():
    import xlb_biot_b200.api as G
    from xlb_biot_b200 import autotune
    saved = autotune.get_config(autotune.ELASTICITY)
    try:
        autotune.set_config(autotune.ELASTICITY, 128, 1, 1, 8, 4)
        big, small = _elasticity(G, 256, 256), _elasticity(G, 128, 128)
        fb, fs = big._L(0).zeros(8), small._L(0).zeros(8)
        assert big._sweep(fb, 0, 0.25, 0.75, query=True) == 4
        assert big._sweep(fb, 0, 1.0, -1.0, sumsq=True, query=True) == 3      # fused sum
        assert small._sweep(fs, 0, 0.25, 0.75, query=True) == 3               # 16 K cells
    finally:
        autotune.set_config(autotune.ELASTICITY, **saved)
