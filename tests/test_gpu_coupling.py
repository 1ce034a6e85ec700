"""The fused Biot coupling force (``xlbb_elast_divgrad``) against the
divergence kernel followed by the gradient kernel: bit for bit, on every
multigrid level, in FP32 and FP64, with and without a base force, for the
walled consolidation problem (gradient boundary rules, per-cell material) and
for a periodic problem whose coarse levels are smaller than one 32 x 8 tile."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _check(el, da, seed):
    for level in range(el.levels):
        L = el._L(level)
        g = torch.Generator(device="cpu").manual_seed(seed + level)
        f = L.field(torch.randn(L.nx, L.ny, 8, generator=g, dtype=torch.float64), 8)
        base = L.field(torch.randn(L.nx, L.ny, 2, generator=g, dtype=torch.float64), 2)
        for b in (None, base):
            ref = da.gradient(el.update_divergence(f, level), 0.37, base=b, dtype=L.dtype)
            got = el.coupling_force(f, level, da, 0.37, base=b)
            assert torch.equal(ref, got), (level, L.nx, L.ny, b is None)


@pytest.mark.parametrize("prec", ["f32/f32", "f64/f64"])
def test_coupling_force_walled_heterogeneous(prec):
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import terzaghi_heterogeneous
    sim, _ = terzaghi_heterogeneous(G, nx=64, ny=34, levels=2, cycles=1, ell=5.0, precision=prec)
    assert sim.elasticity.material_fields(0)[1] is not None
    _check(sim.elasticity, sim.darcy, 1)


@pytest.mark.parametrize("prec", ["f32/f32", "f64/f64"])
def test_coupling_force_periodic_down_to_tiny_levels(prec):
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import periodic_biot_1024
    sim = periodic_biot_1024(G, n=64, levels=5, precision=prec, darcy_precision=prec)
    assert sim.elasticity.grid_size(4) == (4, 4)
    _check(sim.elasticity, sim.darcy, 7)
