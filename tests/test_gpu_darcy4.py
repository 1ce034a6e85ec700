"""The four-column Darcy sweep (launch pipeline 4: a lane takes four cells,
16-byte loads and stores, streaming along x by warp shuffles and recomputed
segment-edge cells) against the collide-and-push sweep (pipeline 3): bitwise
the same populations on

* the headline workload's set-up (log-normal per-cell omega, corner-patched
  anti-bounce-back and bounce-back walls), 256^2 and a width that leaves a
  partial last segment;
* every example Darcy set-up (periodic, anti-bounce-back, equilibrium,
  Neumann bounce-back) with its source plane and an external source;
* grids of one and two lanes per row (the segment's edge cells are both in
  one lane, or in neighbouring lanes);

and the sweeps it does not take (FP64, a fused sum, widths that are not a
multiple of 4) stay on the other pipelines.
"""
import numpy as np
import pytest
import torch

from problems import make_darcy

pytestmark = pytest.mark.gpu


@pytest.fixture
def pipeline():
    from xlb_biot_b200 import autotune
    saved = autotune.get_config(autotune.DARCY)

    def use(p):
        autotune.set_config(autotune.DARCY, 128, 1, 1, 8, p)
    yield use
    autotune.set_config(autotune.DARCY, **saved)


def _sweeps(s, n, ext=None):
    f = s.assign_fields_sharded()
    for t in range(n):
        f, _ = s.step(f, t, external_source=ext)
    torch.cuda.synchronize()
    return f.cpu().numpy()


def _both(pipeline, make, n=8, ext=None):
    out = []
    for p in (3, 4):
        pipeline(p)
        out.append(_sweeps(make(), n, ext))
    return out


@pytest.mark.parametrize("n", [256, 200])
def test_lognormal_workload_bitwise(pipeline, n):
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import darcy_lognormal
    a, b = _both(pipeline, lambda: darcy_lognormal(G, n=n, ell=8.0, precision="f32/f32")[0], n=10)
    assert np.isfinite(a).all() and np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["periodic", "anti", "eq", "neumann"])
@pytest.mark.parametrize("nx,ny", [(200, 36), (4, 12), (8, 10), (132, 5)])
def test_example_setups_bitwise(pipeline, kind, nx, ny):
    import xlb_biot_b200.api as G
    ext = 1e-3 * np.random.default_rng(5).standard_normal((nx, ny, 1))

    def make():
        return make_darcy(G, kind)(lattice=G.LatticeD2Q9("f32/f32"), omega=1.0 / (3 * 0.1 + 0.5), nx=nx, ny=ny,
                                   nz=0, precision="f32/f32", print_info_rate=0)
    a, b = _both(pipeline, make, n=6, ext=ext)
    assert np.isfinite(a).all() and np.array_equal(a, b), kind


def test_pipeline_query_and_fallbacks(pipeline):
    """With pipeline 4 configured, FP32 sweeps of widths divisible by 4 take the
    four-column kernel; FP64 and other widths keep the collide-and-push one."""
    import xlb_biot_b200.api as G
    pipeline(4)
    for prec, nx, want in (("f32/f32", 200, 4), ("f64/f64", 200, 3), ("f32/f32", 202, 3)):
        s = make_darcy(G, "anti")(lattice=G.LatticeD2Q9(prec), omega=1.2, nx=nx, ny=20, nz=0, precision=prec,
                                  print_info_rate=0)
        assert s.sweep_pipeline() == want, (prec, nx)
