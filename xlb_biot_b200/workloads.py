"""Synthetic benchmark workloads (seeded), built against any namespace that
exposes the reference's class names.

* ``darcy_lognormal``: D2Q9 Darcy flow on an ``n x n`` grid, permeability
  ``k = exp(g)`` with ``g`` a Gaussian random field (squared-exponential
  covariance, correlation length ``ell`` cells, unit variance, FFT spectral
  synthesis, numpy seed), per-cell ``omega = 1/(3k + 1/2)``; pressure 1 on the
  left wall and 0 on the right wall (ADR anti-bounce-back), no flux at the
  bottom and top walls (ADR bounce-back), corner directions patched as in the
  reference's Terzaghi example.
"""
import numpy as np


def gaussian_random_field(nx, ny, ell, sigma=1.0, seed=0):
    """Periodic GRF with covariance sigma^2 exp(-r^2 / (2 ell^2)) by spectral
    synthesis, normalised to zero mean and standard deviation ``sigma``."""
    rng = np.random.default_rng(seed)
    kx = 2 * np.pi * np.fft.fftfreq(nx)
    ky = 2 * np.pi * np.fft.fftfreq(ny)
    k2 = kx[:, None] ** 2 + ky[None, :] ** 2
    amp = np.exp(-0.25 * k2 * ell ** 2)             # sqrt of the SE spectral density
    noise = rng.standard_normal((nx, ny)) + 1j * rng.standard_normal((nx, ny))
    g = np.real(np.fft.ifft2(noise * amp))
    g = (g - g.mean()) / g.std()
    return sigma * g


def _corner_patched(m):
    """ADR BCs with the corner-direction patch of the reference's
    ``examples/poroelasticity/Terzaghi.py:22-81`` (a mask mutation inside
    ``get_missing_indices``), generalised to corners on any side."""
    def patch(base):
        class Patched(base):
            def get_missing_indices(self, boundaryMask):
                nbd = len(self.indices[0])
                imissing = np.vstack([np.arange(self.lattice.q, dtype='uint8')] * nbd)
                iknown = np.vstack([np.asarray(self.lattice.opp_indices)] * nbd)
                corners = {(1, 0): (1, 4), (1, self.ny - 1): (2, 8),
                           (self.nx - 2, 0): (1, 7), (self.nx - 2, self.ny - 1): (2, 5)}
                for i in range(nbd):
                    key = (int(self.indices[0][i]), int(self.indices[1][i]))
                    for d in corners.get(key, ()):
                        boundaryMask[i, d] = False
                imissing[~boundaryMask] = 0
                iknown[~boundaryMask] = 0
                return imissing, iknown
        return Patched
    return patch(m.ADR_Neumann_BounceBack), patch(m.ADR_AntiBounceBack)


def darcy_lognormal(m, n=1024, ell=16.0, sigma=1.0, seed=0, precision="f32/f32"):
    """Construct the workload's solver in namespace ``m``.  Returns
    ``(solver, k_field)``; the solver carries the per-cell omega field
    (``omega_field`` keyword of the product, an ``omega`` array in the oracle)."""
    k = np.exp(gaussian_random_field(n, n, ell, sigma, seed))[..., None]
    omega = 1.0 / (3.0 * k + 0.5)
    BB, AntiBB = _corner_patched(m)

    class LognormalDarcy(m.AdvectionDiffusionReactionBGK):
        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            self.BCs.append(AntiBB(tuple(bb["left"].T), self.gridInfo, self.precisionPolicy,
                                   rho=np.ones((len(bb["left"]), 1))))
            self.BCs.append(AntiBB(tuple(bb["right"].T), self.gridInfo, self.precisionPolicy,
                                   rho=np.zeros((len(bb["right"]), 1))))
            self.BCs.append(BB(tuple(bb["bottom"].T), self.gridInfo, self.precisionPolicy))
            self.BCs.append(BB(tuple(bb["top"].T), self.gridInfo, self.precisionPolicy))

    kw = dict(lattice=m.LatticeD2Q9(precision), omega=float(np.mean(omega)), nx=n, ny=n, nz=0,
              precision=precision, print_info_rate=0)
    try:
        solver = LognormalDarcy(omega_field=omega, **kw)
    except TypeError:
        solver = LognormalDarcy(**kw)
    if getattr(solver, "omega_field", None) is None:
        solver.omega = omega.astype(solver.precisionPolicy.compute_dtype)
    return solver, k
