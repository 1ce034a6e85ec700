"""The hand-written adjoint kernels against their forward kernels (FP64).

For each forward map F (affine in its field inputs for fixed material) and
random x, y:  <F(x) - F(0), y> == <x, F^T y>  to rounding, through the C ABI,
on grids with boundary rules of both phases and per-cell material.  The
per-cell parameter gradients are checked against central finite differences
of <F(x; p + eps dp), y> along random directions dp.
"""
import numpy as np
import pytest
import torch

from problems import elastic_material, make_walled_elasticity

pytestmark = pytest.mark.gpu
LAM, MU = elastic_material()


@pytest.fixture(scope="module")
def G():
    import xlb_biot_b200.api as api
    return api


def ip(a, b):
    return float((a.double() * b.double()).sum())


def rnd(L, c, seed, scale=1.0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return L.field(scale * torch.randn(L.nx, L.ny, c, generator=g, dtype=torch.float64), c)


def _hetero_walled(G, kind, nx=34, ny=34, levels=2):
    rng = np.random.default_rng(7)
    lam = LAM * rng.uniform(0.7, 1.3, (nx, ny))
    mu = MU * rng.uniform(0.7, 1.3, (nx, ny))
    kw = dict(**{"lambda": LAM}, mu=MU, nx=nx, ny=ny, nz=0, MG_levels=levels, lambda_field=lam, mu_field=mu,
              MG_BCs={"top": True, "bottom": True, "left": True, "right": True})
    return make_walled_elasticity(G, kind)(lattice=G.LatticeD2Q8("f64/f64"), precision="f64/f64", **kw)


def _fd(set_field, base, d, eps, value):
    vals = []
    for sgn in (1.0, -1.0):
        set_field(base + sgn * eps * d)
        vals.append(value())
    set_field(base)
    return (vals[0] - vals[1]) / (2 * eps)


@pytest.mark.parametrize("kind", ["dirichlet", "neumann"])
@pytest.mark.parametrize("level,a,b,resid", [(0, 0.0, 1.0, False), (0, 0.25, 0.75, False), (0, 1.0, -1.0, False),
                                             (1, 0.25, 0.75, True), (1, 1.0, -1.0, True)])
def test_elast_sweep_adjoint_is_the_transpose(G, kind, level, a, b, resid):
    from xlb_biot_b200.adjoint import ElastGrads, elast_sweep_adjoint
    el = _hetero_walled(G, kind)
    L = el._L(level)
    f, fe, y = rnd(L, 8, 1), rnd(L, 2, 2), rnd(L, 8, 3)
    r = rnd(L, 8, 4) if resid else None
    z8, z2 = L.zeros(8), L.zeros(2)
    out = el._sweep(f, level, a, b, resid=r, fext=fe)
    out0 = el._sweep(z8, level, a, b, resid=z8 if resid else None, fext=z2)
    lhs = ip(out - out0, y)
    lam_r = L.zeros(8) if resid else None
    lam_f, lam_F = elast_sweep_adjoint(el, level, y, a, b, lam_resid=lam_r, want_force=True)
    rhs = ip(f, lam_f) + ip(fe, lam_F) + (ip(r, lam_r) if resid else 0.0)
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + ip(out, out) ** 0.5 * ip(y, y) ** 0.5), (lhs, rhs)

    # parameter gradients of <F(x), y> w.r.t. this level's lambda and mu fields
    grads = ElastGrads(el)
    elast_sweep_adjoint(el, level, y, a, b, f_in=f, resid=r, fext=fe, grads=grads)
    lam_l, mu_l = el.material_fields(level)
    for name, fld, gbuf in (("lambda", lam_l, grads.lam[level]), ("mu", mu_l, grads.mu[level])):
        d = rnd(L, 1, 11)
        base = fld.clone()
        eps = 1e-6 * float(base.abs().max())
        fd = _fd(fld.copy_, base, d, eps, lambda: ip(el._sweep(f, level, a, b, resid=r, fext=fe), y))
        ad = ip(gbuf, d)
        assert abs(fd - ad) <= 1e-6 * abs(fd) + 1e-12, (name, fd, ad)


def _darcy(G):
    from xlb_biot_b200.workloads import darcy_lognormal
    da, _ = darcy_lognormal(G, n=32, ell=4.0, precision="f64/f64")
    return da


def test_darcy_sweep_adjoint_is_the_transpose(G):
    from xlb_biot_b200.adjoint import darcy_sweep_adjoint, f64_plane
    da = _darcy(G)
    L = da._layout
    f, s, y = rnd(L, 9, 1), rnd(L, 1, 2, 0.1), rnd(L, 9, 3)
    out = da._sweep(f, s)
    out0 = da._sweep(L.zeros(9), L.zeros(1))
    lhs = ip(out - out0, y)
    lam_f, lam_s = darcy_sweep_adjoint(da, y, want_source=True)
    rhs = ip(f, lam_f) + ip(s, lam_s)
    assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + ip(out, out) ** 0.5 * ip(y, y) ** 0.5), (lhs, rhs)
    g_om = f64_plane(L)
    darcy_sweep_adjoint(da, y, f_in=f, source=s, g_omega=g_om)
    d = rnd(L, 1, 5)
    fd = _fd(da.omega_field.copy_, da.omega_field.clone(), d, 1e-7, lambda: ip(da._sweep(f, s), y))
    assert abs(fd - ip(g_om, d)) <= 1e-6 * abs(fd), (fd, ip(g_om, d))


@pytest.mark.parametrize("shape", [(32, 18), (16, 10)])
def test_gradient_adjoint_is_the_transpose(G, shape):
    """The Darcy gradient stencil with the consolidation problem's rules (full
    grid) and the fine-level rules restricted to a coarse grid."""
    from xlb_biot_b200.adjoint import gradient_adjoint
    from xlb_biot_b200.fields import Layout
    from xlb_biot_b200.workloads import terzaghi_heterogeneous
    sim, _ = terzaghi_heterogeneous(G, nx=32, ny=18, levels=2, cycles=1, ell=5.0, precision="f64/f64")
    da = sim.darcy
    L = Layout(shape[0], shape[1], torch.float64)
    q, y = rnd(L, 1, 1), rnd(L, 2, 2)
    out = da.gradient(q, 0.37)
    out0 = da.gradient(L.zeros(1), 0.37)
    lhs = ip(out - out0, y)
    lq = L.zeros(1)
    gradient_adjoint(da, y, 0.37, lq)
    assert abs(lhs - ip(q, lq)) <= 1e-12 * (abs(lhs) + ip(out, out) ** 0.5 * ip(y, y) ** 0.5)


def test_moment_adjoints_are_the_transposes(G):
    from xlb_biot_b200.adjoint import ElastGrads, darcy_moments_adjoint, elast_moments_adjoint, f64_plane
    el = _hetero_walled(G, "neumann")
    L = el._L(0)
    f, yd, ye = rnd(L, 8, 1), rnd(L, 1, 2), rnd(L, 2, 3)
    div = el.update_divergence(f, 0)
    eta, _ = el.update_macroscopic(f)
    eta0, _ = el.update_macroscopic(L.zeros(8))
    lhs = ip(div, yd) + ip(eta - eta0, ye)
    lam_f = L.zeros(8)
    elast_moments_adjoint(el, 0, lam_f, lam_eta=ye, lam_div=yd)
    assert abs(lhs - ip(f, lam_f)) <= 1e-12 * (abs(lhs) + 1.0)
    grads = ElastGrads(el)
    elast_moments_adjoint(el, 0, L.zeros(8), lam_div=yd, f=f, grads=grads)
    _, mu_l = el.material_fields(0)
    d = rnd(L, 1, 9)
    base = mu_l.clone()
    fd = _fd(mu_l.copy_, base, d, 1e-6 * float(base.abs().max()), lambda: ip(el.update_divergence(f, 0), yd))
    assert abs(fd - ip(grads.mu[0], d)) <= 1e-6 * abs(fd)

    da = _darcy(G)
    Ld = da._layout
    f9, yr, yg = rnd(Ld, 9, 1), rnd(Ld, 1, 2), rnd(Ld, 2, 3)
    rho, grad = da.update_macroscopic(f9, gradient=True)
    lhs = ip(rho, yr) + ip(grad, yg)
    lam = Ld.zeros(9)
    darcy_moments_adjoint(da, lam, lam_rho=yr, lam_grad=yg)
    assert abs(lhs - ip(f9, lam)) <= 1e-12 * (abs(lhs) + 1.0)
    g_om = f64_plane(Ld)
    darcy_moments_adjoint(da, Ld.zeros(9), lam_grad=yg, f=f9, g_omega=g_om)
    d = rnd(Ld, 1, 4)
    fd = _fd(da.omega_field.copy_, da.omega_field.clone(), d, 1e-7,
             lambda: ip(da.update_macroscopic(f9, gradient=True)[1], yg))
    assert abs(fd - ip(g_om, d)) <= 1e-6 * abs(fd)


def test_fused_divgrad_adjoint_equals_composition(G):
    """xlbb_divgrad_adjoint (one kernel) equals the gradient-stencil transpose
    followed by the divergence transpose, plus the force accumulation."""
    from xlb_biot_b200.adjoint import ElastGrads, divgrad_adjoint, elast_moments_adjoint, gradient_adjoint
    from xlb_biot_b200.workloads import terzaghi_heterogeneous
    sim, _ = terzaghi_heterogeneous(G, nx=32, ny=18, levels=2, cycles=1, ell=5.0, precision="f64/f64")
    el, da = sim.elasticity, sim.darcy
    for level in range(el.levels):
        L = el._L(level)
        lam_ext, f = rnd(L, 2, 1), rnd(L, 8, 2)
        g1, g2 = ElastGrads(el), ElastGrads(el)
        a_f, a_fe = rnd(L, 8, 3), rnd(L, 2, 4)
        b_f, b_fe = L.empty(8), L.empty(2)
        b_f.copy_(a_f)
        b_fe.copy_(a_fe)
        divgrad_adjoint(el, da, level, lam_ext, 0.3, a_f, lam_fe=a_fe, f=f, grads=g1)
        lam_div = L.zeros(1)
        gradient_adjoint(da, lam_ext, 0.3, lam_div, dtype=L.dtype)
        elast_moments_adjoint(el, level, b_f, lam_div=lam_div, f=f, grads=g2)
        b_fe.add_(lam_ext)
        for x, y in ((a_f, b_f), (a_fe, b_fe), (g1.mu[level], g2.mu[level]), (g1.lam[level], g2.lam[level])):
            assert torch.allclose(x, y, rtol=1e-13, atol=1e-13 * float(y.abs().max()))
