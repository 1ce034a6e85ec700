"""Synthetic benchmark workloads (seeded), built against any namespace that
exposes the reference's class names.

* ``darcy_lognormal``: D2Q9 Darcy flow on an ``n x n`` grid, permeability
  ``k = exp(g)`` with ``g`` a Gaussian random field (squared-exponential
  covariance, correlation length ``ell`` cells, unit variance, FFT spectral
  synthesis, numpy seed), per-cell ``omega = 1/(3k + 1/2)``; pressure 1 on the
  left wall and 0 on the right wall (ADR anti-bounce-back), no flux at the
  bottom and top walls (ADR bounce-back), corner directions patched as in the
  reference's Terzaghi example.
* ``lid_driven_cavity``: the D2Q9 fluid cavity of ``MLUPS2d.py``.
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


def manufactured_elasticity(n, lam, mu):
    """Displacement u = (sin 2pi x sin 2pi y, cos 2pi x sin 2pi y) on cell centres
    x = (i + 1/2)/n and the body force eps^2 (-div sigma(u)), eps = 1/n, of plane
    linear elasticity sigma = lam tr(e) I + 2 mu e (the convention of the
    reference's periodic example).  Returns (u, force) of shape (n, n, 2)."""
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    s, c = np.sin(2 * np.pi * X), np.cos(2 * np.pi * X)
    sy, cy = np.sin(2 * np.pi * Y), np.cos(2 * np.pi * Y)
    u = np.stack((s * sy, c * sy), axis=-1)
    k2 = 4 * np.pi ** 2
    # -div sigma = -(lam + mu) grad(div u) - mu lap(u)
    fx = (lam + mu) * k2 * (s * sy + s * cy) + 2 * k2 * mu * s * sy
    fy = -(lam + mu) * k2 * (c * cy - c * sy) + 2 * k2 * mu * c * sy
    return u, np.stack((fx, fy), axis=-1) / n ** 2


def plain_elasticity_128(m, n=128, lam=1.0, mu=1.0, precision="f32/f32"):
    """Plain D2Q8 elasticity on an n x n periodic grid with the manufactured
    force (no multigrid); populations start at zero."""
    u, force = manufactured_elasticity(n, lam, mu)

    class Manufactured(m.LBMElasticity):
        def get_force(self):
            return self.distributed_array_init((n, n, 2), self.precisionPolicy.compute_dtype, init_val=force)

        def initialize_macroscopic_fields(self):
            return None, None

    solver = Manufactured(lattice=m.LatticeD2Q8(precision), **{"lambda": lam}, mu=mu, nx=n, ny=n, nz=0,
                          precision=precision, print_info_rate=0)
    return solver, u


EXAMPLE_E, EXAMPLE_NU = 0.11, 0.8     # material of the reference's periodic examples


def periodic_biot_1024(m, n=1024, levels=5, lam=None, mu=None, alpha=1.0, K=0.1, precision="f32/f32",
                       darcy_precision=None, coarsest_precision=None, tol=None, max_cycles=8,
                       residual_precision=None):
    """Periodic Biot consolidation with the initial pressure sin 2pi x sin 2pi y:
    elasticity with an L-level V-cycle per time step (``max_cycles`` cycles, or
    until the residual fell by ``tol``), Darcy with K = 0.1 (omega = 1.25),
    alpha = 1, centred coupling.  The default material is the one of the
    reference's periodic examples (E = 0.11, nu = 0.8, plane stress); with
    lam = 2, mu = 1 in lattice units the reference's V-cycle diverges.  The
    storativity enters through the pressure unit (p in units of 1/c0)."""
    if lam is None:
        lam = EXAMPLE_E * EXAMPLE_NU / (1 - EXAMPLE_NU ** 2)
    if mu is None:
        mu = 0.5 * EXAMPLE_E / (1 + EXAMPLE_NU)
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    p0 = (np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y))[..., None]

    class PD(m.AdvectionDiffusionReactionBGK):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((n, n, 1), self.precisionPolicy.output_dtype, init_val=p0),
                    self.distributed_array_init((n, n, 2), self.precisionPolicy.output_dtype, init_val=0.0))

    class PE(m.LBMElasticity):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((n, n, 2), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((n, n, 3), self.precisionPolicy.output_dtype, init_val=0.0))

    class PB(m.LBMPoroelasticity):
        def __init__(self, **kw):
            super().__init__(PE, PD, **kw)

    kw = dict(lattice_elasticity=m.LatticeD2Q8(precision), lattice_darcy=m.LatticeD2Q9(darcy_precision or precision),
              **{"lambda": lam}, mu=mu, omega=1.0 / (3 * K + 0.5), alpha=alpha, nx=n, ny=n, nz=0,
              precision=precision, elasticity_MG_levels=levels, elasticity_steps=max_cycles,
              coupling_method="centered", print_info_rate=0)
    if darcy_precision:
        kw["darcy_precision"] = darcy_precision
    if coarsest_precision:
        kw["coarsest_precision"] = coarsest_precision
    if tol is not None:
        kw["elasticity_tol"] = tol
    if residual_precision:
        kw["residual_precision"] = residual_precision
    return PB(**kw)


def fourier_force(n, rng, modes=4):
    """Sum of ``modes`` periodic Fourier modes with N(0, 1) amplitudes (random
    wave numbers 1..3, phases), scaled by 1/n^2 like the examples' forces."""
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x, indexing="ij")
    f = np.zeros((n, n, 2))
    for _ in range(modes):
        kx, ky = rng.integers(1, 4, size=2)
        ph = rng.uniform(0, 2 * np.pi, size=2)
        a = rng.standard_normal(2)
        arg = 2 * np.pi * (kx * X + ky * Y)
        f[..., 0] += a[0] * np.sin(arg + ph[0])
        f[..., 1] += a[1] * np.cos(arg + ph[1])
    return f / n ** 2


def batch_instances(count=512, sizes=(64, 96, 128, 192, 256, 384), mu_range=(0.5, 2.0), nu_range=(0.1, 0.4),
                    stress_unit=16.0, seed=0):
    """Seeded heterogeneous batch: square sizes drawn uniformly from ``sizes``,
    shear modulus uniform in ``mu_range`` and Poisson ratio uniform in
    ``nu_range`` (plane stress, lam = 2 mu nu / (1 - nu)), random smooth
    forces.  Moduli are expressed in units of ``stress_unit``: the D2Q8
    model's equilibrium is singular at lattice lambda + mu = 1/3 and the
    reference's V-cycle diverges for lattice moduli of order one, so the
    default keeps lambda + mu <= 0.29."""
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.asarray(sizes), size=count)
    mus = rng.uniform(*mu_range, size=count) / stress_unit
    nus = rng.uniform(*nu_range, size=count)
    lams = 2 * mus * nus / (1 - nus)
    forces = [fourier_force(int(n), rng) for n in ns]
    return [(int(n), int(n)) for n in ns], lams, mus, forces


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


# Non-dimensional material of the reference's 2D consolidation example
# (examples/poroelasticity/2D.py: E = 1e5, nu = 0.9 plane-stress Lame
# parameters, c0 = 1e-6, kappa = 1e-9, L = 100, T = 2e6, load 1e4), which in
# lattice units does not depend on nx except through epsilon and the load.
TERZAGHI_LAM = 0.1 * 0.9 / (1 - 0.9 ** 2)
TERZAGHI_MU = 0.5 * 0.1 / (1 + 0.9)
TERZAGHI_K = 0.2


def terzaghi_heterogeneous(m, nx=512, ny=258, levels=5, mu0=TERZAGHI_MU, lam0=TERZAGHI_LAM, nu=None,
                           K0=TERZAGHI_K, sigma=0.5, ell=24.0, load=None, epsilon=None, cycles=4, k_smooth=4,
                           seed=0, precision="f32/f32", darcy_precision=None, coarsest_precision=None,
                           residual_precision=None, log_mu=None, log_k=None):
    """2D Terzaghi-type consolidation with heterogeneous material.

    A layer of ``ny - 2`` cell rows (plus one boundary row at the bottom and at
    the top), periodic in x (laterally infinite: no net flux through the
    sides).  Elasticity: fixed bottom (full-way bounce-back), top loaded by the
    traction (0, -load * (1 - cos(2 pi (x + 1/2) / nx)) / 2) (anti-bounce-back);
    Darcy: no flux at the bottom (bounce-back), drained top p = 0
    (anti-bounce-back); zero initial displacement and pressure.  Per-cell
    shear modulus mu = mu0 exp(g_mu) with lambda = lam0 (or, if ``nu`` is
    given, lambda = 2 mu nu / (1 - nu) per cell), permeability
    K = K0 exp(g_K), omega = 1 / (3 K + 1/2); g_mu, g_K seeded Gaussian random
    fields (correlation length ``ell``, standard deviation ``sigma``) unless
    given (``log_mu``, ``log_k``: the fields g).  Defaults: the reference's 2D
    example in lattice units (epsilon = 100 / nx, load = 1 / nx).
    ``levels``-level V-cycles (MG_BCs bottom/top, ``k_smooth`` smoothing
    sweeps), ``cycles`` V-cycles per time step, centred coupling.
    Returns (sim, material) with material = dict(log_mu, log_k, mu, lam, K, omega)."""
    load = 1.0 / nx if load is None else load
    epsilon = 100.0 / nx if epsilon is None else epsilon
    g_mu = gaussian_random_field(nx, ny, ell, sigma, seed) if log_mu is None else np.asarray(log_mu, np.float64)
    g_k = gaussian_random_field(nx, ny, ell, sigma, seed + 1) if log_k is None else np.asarray(log_k, np.float64)
    mu = mu0 * np.exp(g_mu)
    lam = mu * (2 * nu / (1 - nu)) if nu is not None else np.full_like(mu, lam0)
    K = K0 * np.exp(g_k)
    omega = 1.0 / (3.0 * K + 0.5)
    x = np.arange(nx)
    traction = np.zeros((nx, 2))
    traction[:, 1] = -load * 0.5 * (1 - np.cos(2 * np.pi * (x + 0.5) / nx))

    class Darcy(m.AdvectionDiffusionReactionBGK):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((self.nx, self.ny, 1), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0))

        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            self.BCs.append(m.ADR_Neumann_BounceBack(tuple(bb["bottom"].T), self.gridInfo, self.precisionPolicy))
            self.BCs.append(m.ADR_AntiBounceBack(tuple(bb["top"].T), self.gridInfo, self.precisionPolicy,
                                                 rho=np.zeros((len(bb["top"]), 1))))

    class Elasticity(m.LBMElasticity):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((self.nx, self.ny, 3), self.precisionPolicy.output_dtype, init_val=0.0))

        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            self.BCs.append(m.ElasticityBounceBackFullway(tuple(bb["bottom"].T), self.gridInfo, self.precisionPolicy))
            self.BCs.append(m.ElasticityAntiBounceBack(tuple(bb["top"].T), self.gridInfo, self.precisionPolicy,
                                                       traction))
            for level in range(1, self.levels):
                gi, bbl = self.grid_info(level), self.bounding_box_indices(level)
                self.BCs_MG[level] = [
                    m.ElasticityBounceBackFullway(tuple(bbl["bottom"].T), gi, self.precisionPolicy),
                    m.ElasticityAntiBounceBack(tuple(bbl["top"].T), gi, self.precisionPolicy)]

    class Consolidation(m.LBMPoroelasticity):
        def __init__(self, **kw):
            super().__init__(Elasticity, Darcy, **kw)

    kw = dict(lattice_elasticity=m.LatticeD2Q8(precision), lattice_darcy=m.LatticeD2Q9(darcy_precision or precision),
              **{"lambda": float(np.mean(lam))}, mu=float(np.mean(mu)), lambda_field=lam, mu_field=mu,
              omega=float(np.mean(omega)), omega_field=omega[..., None], alpha=1.0, epsilon=float(epsilon),
              nx=nx, ny=ny, nz=0,
              precision=precision, elasticity_MG_levels=levels, elasticity_steps=cycles,
              MG_BCs={"bottom": True, "top": True}, MG_n_smoothing=k_smooth, coupling_method="centered",
              print_info_rate=0)
    if darcy_precision:
        kw["darcy_precision"] = darcy_precision
    if coarsest_precision:
        kw["coarsest_precision"] = coarsest_precision
    if residual_precision:
        kw["residual_precision"] = residual_precision
    sim = Consolidation(**kw)
    if getattr(sim.darcy, "omega_field", None) is None:
        sim.darcy.omega = omega[..., None].astype(sim.darcy.precisionPolicy.compute_dtype)
    return sim, dict(log_mu=g_mu, log_k=g_k, mu=mu, lam=lam, K=K, omega=omega)


def lid_driven_cavity(m, model="bgk", u_wall=0.1, Re=100.0):
    """The fluid workload of ``examples/performance/MLUPS2d.py``: lid-driven
    cavity with full-way bounce-back on the left, right and bottom walls and
    the equilibrium of (rho = 1, u = (u_wall, 0)) on the top row.  Returns the
    solver class (``m.BGKSim`` or ``m.KBCSim`` based) and ``omega(n)`` from
    ``Re`` with the example's characteristic length n - 1."""
    base = m.BGKSim if model == "bgk" else m.KBCSim

    class Cavity(base):
        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            walls = np.concatenate((bb["left"], bb["right"], bb["bottom"]))
            self.BCs.append(m.BounceBack(tuple(walls.T), self.gridInfo, self.precisionPolicy))
            lid = bb["top"]
            dt = self.precisionPolicy.compute_dtype
            rho_wall = np.ones((lid.shape[0], 1), dtype=dt)
            vel_wall = np.zeros(lid.shape, dtype=dt)
            vel_wall[:, 0] = u_wall
            self.BCs.append(m.EquilibriumBC(tuple(lid.T), self.gridInfo, self.precisionPolicy, rho_wall, vel_wall))

    def omega(n):
        return 1.0 / (3.0 * (u_wall * (n - 1) / Re) + 0.5)
    return Cavity, omega


def lid_driven_cavity_3d(m, u_wall=0.1, Re=100.0, model="bgk"):
    """The fluid workload of ``examples/performance/MLUPS3d.py``: a cubic
    cavity with full-way bounce-back on the left, right, bottom, front and back
    faces and the equilibrium of (rho = 1, u = (u_wall, 0, 0)) on the top face
    (z = nz - 1); BGK collision as the example (``model="kbc"``: the KBC
    collision, D3Q27 only).  Returns the solver class and ``omega(n)``."""
    base = m.BGKSim if model == "bgk" else m.KBCSim

    class Cavity3D(base):
        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            walls = np.concatenate((bb["left"], bb["right"], bb["bottom"], bb["front"], bb["back"]))
            self.BCs.append(m.BounceBack(tuple(walls.T), self.gridInfo, self.precisionPolicy))
            lid = bb["top"]
            dt = self.precisionPolicy.compute_dtype
            rho_wall = np.ones((lid.shape[0], 1), dtype=dt)
            vel_wall = np.zeros(lid.shape, dtype=dt)
            vel_wall[:, 0] = u_wall
            self.BCs.append(m.EquilibriumBC(tuple(lid.T), self.gridInfo, self.precisionPolicy, rho_wall, vel_wall))

    def omega(n):
        return 1.0 / (3.0 * (u_wall * (n - 1) / Re) + 0.5)
    return Cavity3D, omega
