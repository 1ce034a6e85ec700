"""Pins of the oracle's D2Q9 fluid models (``src/models.py`` BGK and KBC).

The reference verifies its fluid path only by running it
(``examples/performance/MLUPS2d.py``); the oracle is pinned here by the
analytic decay of a periodic shear wave, u_x = A sin(k y) exp(-nu k^2 t) with
nu = (1/omega - 1/2) / 3, at second order in the grid spacing, by mass
conservation, and by the lid-driven cavity staying finite with the lid speed
imposed on the top row.
"""
import numpy as np
import pytest

import oracle.api as O
from problems import make_cavity, make_shear_wave


def _shear_error(model, n, omega=1.2):
    S = make_shear_wave(O, model)
    s = S(lattice=O.LatticeD2Q9("f64/f64"), omega=omega, nx=4, ny=n, nz=0, precision="f64/f64")
    f = s.assign_fields_sharded()
    m0 = f.sum()
    T = n * n // 8
    for t in range(T):
        f, _ = s.step(f, t)
    _, u = s.update_macroscopic(f)
    nu, k = (1 / omega - 0.5) / 3, 2 * np.pi / n
    ex = 0.02 * np.sin(2 * np.pi * (np.arange(n) + 0.5) / n) * np.exp(-nu * k * k * T)
    assert abs(f.sum() - m0) < 1e-10 * m0
    return np.abs(u[0, :, 0] - ex).max() / np.abs(ex).max(), np.abs(u[..., 1]).max()


@pytest.mark.parametrize("model", ["bgk", "kbc"])
def test_shear_wave_decay_second_order(model):
    e32, v32 = _shear_error(model, 32)
    e64, v64 = _shear_error(model, 64)
    assert e32 < 4e-3 and e64 < 1e-3
    assert 3.5 < e32 / e64 < 4.5
    assert max(v32, v64) < 1e-6


def test_kbc_equals_bgk_at_omega_one_on_pure_shear():
    """With omega = 1 (beta = 1/2) both collisions relax the shear part fully;
    on a flow with no higher-order non-equilibrium the two agree closely."""
    out = []
    for model in ("bgk", "kbc"):
        S = make_shear_wave(O, model)
        s = S(lattice=O.LatticeD2Q9("f64/f64"), omega=1.0, nx=4, ny=32, nz=0, precision="f64/f64")
        f = s.assign_fields_sharded()
        for t in range(20):
            f, _ = s.step(f, t)
        out.append(s.update_macroscopic(f)[1])
    assert np.abs(out[0] - out[1]).max() < 1e-4 * np.abs(out[0]).max()


@pytest.mark.parametrize("model", ["bgk", "kbc"])
def test_cavity_runs_and_imposes_the_lid(model):
    C, om = make_cavity(O, model)
    s = C(lattice=O.LatticeD2Q9("f64/f64"), omega=om(24), nx=24, ny=24, nz=0, precision="f64/f64")
    f = s.run(100)
    rho, u = s.update_macroscopic(f)
    assert np.isfinite(f).all()
    np.testing.assert_allclose(u[:, -1, 0], 0.1, rtol=1e-12)
    assert u[1:-1, -2, 0].mean() > 0.02           # the lid drags the fluid below it
    assert u[1:-1, 1:-2, 0].min() < 0             # and drives a recirculation


def _cavity_ulp_sensitivity(model, prec, eps):
    C, om = make_cavity(O, model)
    outs = []
    for pert in (0.0, eps):
        s = C(lattice=O.LatticeD2Q9(prec), omega=om(64), nx=64, ny=48, nz=0, precision=prec)
        f = s.assign_fields_sharded()
        f = (f * (1 + pert * np.random.default_rng(0).standard_normal(f.shape))).astype(f.dtype)
        for t in range(61):
            f, _ = s.step(f, t)
        outs.append(f.astype(np.float64))
    return np.abs(outs[0] - outs[1]).max() / np.abs(outs[0]).max()


def test_kbc_cavity_is_ill_conditioned_in_rounding():
    """The tolerance of the GPU KBC cavity comparison: a one-ulp perturbation of
    the initial populations moves the oracle's own 61-step KBC cavity by about
    1e-12 (FP64), against 2e-15 for BGK, because gamma divides by <dH, dH>."""
    bgk = _cavity_ulp_sensitivity("bgk", "f64/f64", 1e-16)
    kbc = _cavity_ulp_sensitivity("kbc", "f64/f64", 1e-16)
    assert bgk < 1e-14
    assert 1e-13 < kbc < 1e-10
