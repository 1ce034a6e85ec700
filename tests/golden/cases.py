"""Golden cases: the same seeded set-ups run through any namespace ``m`` that
exposes the reference's class names -- the reference's own modules (fixture
generation, ``make_golden.py``), the oracle (CPU test) or the CUDA product (GPU
test).  Each case returns a dict of NumPy arrays (FP64 runs).

The set-ups are the reference's examples as restated in ``tests/problems.py``:
periodic / walled elasticity (``examples/elasticity/*.py``), the four Darcy
examples (``examples/darcy/*.py``), periodic Biot
(``examples/poroelasticity/periodic.py``) and the corner-patched Terzaghi
consolidation (``examples/poroelasticity/Terzaghi.py``).
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(1, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from problems import (elastic_material, make_darcy, make_periodic_biot, make_periodic_elasticity,  # noqa: E402
                      make_terzaghi, make_walled_elasticity)

PREC = "f64/f64"
LAM, MU = elastic_material()


def to_np(x):
    """Host FP64 copy of a reference/oracle/product array or scalar."""
    if x is None:
        return None
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.array(np.asarray(x), dtype=np.float64)


def _in(m, x):
    """An input array in the namespace's own array type (the reference's
    functional updates need its array class; the oracle and the product take
    NumPy)."""
    conv = getattr(m, "golden_asarray", None)
    return conv(x) if conv is not None else x


def _el(m, cls, prec=PREC, **kw):
    return cls(lattice=m.LatticeD2Q8(prec), **{"lambda": LAM}, mu=MU, nz=0, precision=prec, print_info_rate=0, **kw)


def elast_plain(m, nx, ny, sweeps=20, prec=PREC):
    """Periodic elasticity from a seeded random equilibrium, plain sweeps, then
    the macroscopic fields and the divergence (``src/elasticity.py:1128-1219``,
    ``:1003-1058``)."""
    P = make_periodic_elasticity(m)
    P.init_seed = 3
    s = _el(m, P, prec, nx=nx, ny=ny)
    f = s.assign_fields_sharded()
    out = {"f0": to_np(f)}
    for t in range(sweeps):
        f, _ = s.step(f, t)
    eta, sigma = s.update_macroscopic(f)
    out.update(f=to_np(f), eta=to_np(eta), sigma=to_np(sigma), div=to_np(s.update_divergence(f)))
    return out


def elast_periodic_mg(m, n=32, levels=3, cycles=3):
    """Periodic multigrid V-cycles (``:1221-1312``) with their level-0 residual norms."""
    P = make_periodic_elasticity(m)
    P.init_seed = 5
    s = _el(m, P, nx=n, ny=n, MG_levels=levels)
    f = s.assign_fields_sharded()
    norms = []
    for t in range(cycles):
        f, r = s.step(f, t)
        norms.append(float(to_np(r)))
    return {"f": to_np(f), "norms": np.array(norms)}


def elast_walled_mg(m, kind, cycles=4, prec=PREC):
    """``dirichlet_MG.py`` / ``neumann_MG.py``: BC rules on every level, 3 levels."""
    kw = dict(nx=18, ny=18, MG_levels=3, MG_BCs={"top": True, "bottom": True, "left": True, "right": True})
    s = _el(m, make_walled_elasticity(m, kind), prec, **kw)
    f = 1e-3 * np.random.default_rng(7).standard_normal((18, 18, 8))
    out = {"f0": f.copy()}
    norms = []
    for t in range(cycles):
        f, r = s.step(_in(m, f) if t == 0 else f, t)
        norms.append(float(to_np(r)))
    out.update(f=to_np(f), norms=np.array(norms))
    return out


def elast_halfway(m):
    """``ElasticityBounceBack`` (halfway, wall displacement) on all four sides
    with an external force: the zero-padded missing/known tables
    (``src/elasticity.py:1552-1646``)."""
    class H(m.LBMElasticity):
        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            walls = np.concatenate((bb["left"], bb["right"], bb["top"], bb["bottom"]))
            self.BCs.append(m.ElasticityBounceBack(tuple(walls.T), self.gridInfo, self.precisionPolicy,
                                                   np.array([1e-3, -2e-3])))
    s = _el(m, H, nx=12, ny=10)
    f = np.random.default_rng(1).standard_normal((12, 10, 8))
    out = {"f0": f.copy()}
    ext = _in(m, 0.01 * np.ones((12, 10, 2)))
    f = _in(m, f)
    for t in range(5):
        f, _ = s.step(f, t, external_force=ext)
    out["f"] = to_np(f)
    return out


def darcy(m, kind, sweeps=30, prec=PREC):
    """``examples/darcy/*.py`` set-ups: sweeps with an alternating external
    source, then pressure, pressure gradient and the isotropic gradient
    (``src/darcy.py:36-171``, BCs ``:298-466``)."""
    nx = 24 if kind == "periodic" else 26
    s = make_darcy(m, kind)(lattice=m.LatticeD2Q9(prec), omega=1.0 / (3 * 0.1 + 0.5), nx=nx, ny=nx - 4, nz=0,
                            precision=prec, print_info_rate=0)
    f = s.assign_fields_sharded()
    out = {"f0": to_np(f)}
    ext = _in(m, 1e-3 * np.random.default_rng(2).standard_normal((nx, nx - 4, 1)))
    for t in range(sweeps):
        f, _ = s.step(f, t, external_source=ext if t % 2 else None)
    rho, grad = s.update_macroscopic(f, ext, gradient=True)
    out.update(f=to_np(f), rho=to_np(rho), grad=to_np(grad), gradient=to_np(s.gradient(rho, 0.3)))
    return out


def darcy_cell_omega(m, nx=20, ny=16, sweeps=10):
    """The Darcy sweep with a per-cell relaxation field (heterogeneous
    permeability, the benchmark's variant): the reference's collision
    expressions (``src/darcy.py:118-127``) broadcast an (nx, ny, 1) omega
    array cell by cell."""
    K = np.exp(np.random.default_rng(5).standard_normal((nx, ny, 1)))
    om = 1.0 / (3 * K + 0.5)
    cls = make_darcy(m, "anti")
    kw = dict(lattice=m.LatticeD2Q9(PREC), omega=1.0, nx=nx, ny=ny, nz=0, precision=PREC, print_info_rate=0)
    if getattr(m, "golden_cell_omega", None) == "field":
        s = cls(omega_field=om, **kw)
    else:
        s = cls(**kw)
        m.golden_set_omega(s, _in(m, om))
    f = s.assign_fields_sharded()
    for t in range(sweeps):
        f, _ = s.step(f, t)
    return {"omega": om, "f": to_np(f)}


def _records(sim):
    """The ``output_data`` records of a Biot ``run`` stacked per field."""
    keys = ("eta", "sigma", "pressure", "pressure_grad", "dt_div_eta")
    out = {k: np.stack([to_np(r[k]) for r in sim.records]) for k in keys}
    out["timesteps"] = np.array([int(to_np(r["timestep"])) for r in sim.records], dtype=np.float64)
    return out


def biot_periodic(m, levels, t_max=5):
    """``examples/poroelasticity/periodic.py`` through the reference's ``run``
    (``src/poroelasticity.py:208-301``): dynamic force and source, the coupling
    force inside every smoothing sweep; every step's outputs recorded."""
    K = 0.1
    sim = make_periodic_biot(m)(lattice_elasticity=m.LatticeD2Q8(PREC), lattice_darcy=m.LatticeD2Q9(PREC),
                                **{"lambda": LAM}, mu=MU, omega=1 / (3 * K + 0.5), alpha=1.0, nx=16, ny=16, nz=0,
                                precision=PREC, elasticity_steps=2, elasticity_MG_levels=levels, io_rate=1,
                                print_info_rate=0)
    sim.run(t_max)
    return _records(sim)


def biot_terzaghi(m, t_max=4):
    """``examples/poroelasticity/Terzaghi.py``: corner-patched BC subclasses,
    MG_BCs left/right, four smoothing sweeps, three levels (the coarse levels'
    coupling gradient uses the fine-level Darcy rules, ``:324``)."""
    sim = make_terzaghi(m)(lattice_elasticity=m.LatticeD2Q8(PREC), lattice_darcy=m.LatticeD2Q9(PREC),
                           **{"lambda": LAM}, mu=MU, omega=1.0 / (3 * 0.7 + 0.5), alpha=1.0, nx=18, ny=4, nz=0,
                           precision=PREC, elasticity_steps=2, elasticity_MG_levels=3,
                           MG_BCs={"left": True, "right": True}, MG_n_smoothing=4, epsilon=0.5, io_rate=1,
                           print_info_rate=0)
    sim.run(t_max)
    return _records(sim)


def mg_transfers(m):
    """``_restrict`` (2x2 block sums), ``_prolong`` (injection) and
    ``equilibrium`` with an external force (``src/elasticity.py:851-957``)."""
    kw = dict(nx=18, ny=14, MG_levels=2, MG_BCs={"left": True, "right": True, "bottom": True, "top": True})
    s = _el(m, m.LBMElasticity, **kw)
    rng = np.random.default_rng(11)
    r = rng.standard_normal((18, 14, 8))
    c = rng.standard_normal((10, 8, 8))
    eta, sig, ext = rng.standard_normal((18, 14, 2)), rng.standard_normal((18, 14, 3)), rng.standard_normal((18, 14, 2))
    return {"restrict": to_np(s._restrict(_in(m, r))), "prolong": to_np(s._prolong(_in(m, c))),
            "equilibrium": to_np(s.equilibrium(_in(m, eta), _in(m, sig), external_force=_in(m, ext)))}


PARAMETER_KEYS = ("L_tot", "E", "nu", "c0", "alpha", "lambda", "mu", "force", "Kpm", "p0", "eta0", "etaInf",
                  "kappa", "c_f", "T_tot")


def parameters_terzaghi(m, alpha=0.8):
    """``Parameters`` (``src/utils.py:17-76``) driven as the Terzaghi example
    does (``examples/poroelasticity/Terzaghi.py:247-280``): SI units, derived
    2-D Lame parameters, load, pressures and times, then the non-dimensional
    units L_tot, eta0, T_tot, p0; every parameter's dimensional and
    non-dimensional value, and the type checks of the setters."""
    params = m.Parameters()
    params.add_units(L=1.0, H=1.0, T=1.0, P=1.0)
    params.add_parameters(L_tot=(1e0, {'L': 1}), E=(1.0, {'P': 1}), nu=(0.8, {}), c0=(1e0, {'P': -1}),
                          alpha=(alpha, {}))
    g = params.get
    params.set_parameter('lambda', g('E') * g('nu') / (1 - g('nu') ** 2), {'P': 1})
    params.set_parameter('mu', 0.5 * g('E') / (1 + g('nu')), {'P': 1})
    params.add_parameters(
        force=(g('alpha') / g('c0') + (g('lambda') + 2 * g('mu')) / g('alpha'), {'L': -1, 'H': 1, 'P': 1}),
        Kpm=(g('lambda') + 2 * g('mu') + g('alpha') ** 2 / g('c0'), {'P': 1}))
    params.add_parameters(
        p0=(g('alpha') * g('force') / g('c0') / g('Kpm'), {'P': 1}),
        eta0=(g('force') * g('L_tot') / g('Kpm'), {'H': 1}),
        etaInf=(g('force') * g('L_tot') / (g('lambda') + 2 * g('mu')), {'H': 1}),
        kappa=(g('Kpm') / (g('lambda') + 2 * g('mu')), {'L': 2, 'T': -1, 'P': -1}))
    params.set_parameter('c_f', g('kappa') * (g('lambda') + 2 * g('mu')) / g('c0') / g('Kpm'), {'L': 2, 'T': -1})
    params.set_parameter('T_tot', g('L_tot') ** 2 / g('c_f'), {'T': 1})
    dimensional = [g(k) for k in PARAMETER_KEYS]
    params.add_units(L=g('L_tot'), H=g('eta0'), T=g('T_tot'), P=g('p0'))
    rejected = []
    for bad in (lambda: params.set_unit('L', 1), lambda: params.set_unit('L', -1.0),
                lambda: params.set_parameter('x', 1, {}), lambda: params.set_parameter('x', 1.0, {'Q': 1}),
                lambda: params.set_parameter('x', 1.0, {'L': 1.0}), lambda: params.set_parameter('x', 1.0, [])):
        try:
            bad()
            rejected.append(0.0)
        except TypeError:
            rejected.append(1.0)
    return {"dimensional": np.array(dimensional),
            "nondimensional": np.array([params.get_nondimensional(k) for k in PARAMETER_KEYS]),
            "units": np.array([params.get_unit(k) for k in "LHTP"]), "rejected": np.array(rejected)}


def fluid_cavity(m, model, lattice="D2Q9", n=(24, 20), t_max=20):
    """The cavities of ``examples/performance/MLUPS2d.py`` (BGK and KBC on
    D2Q9) and ``MLUPS3d.py`` (BGK on D3Q19 / D3Q27; KBC on D3Q27) through the reference's
    ``run`` (``src/base.py:848-948``): t_max + 1 steps from rest."""
    from xlb_biot_b200.workloads import lid_driven_cavity, lid_driven_cavity_3d
    if lattice == "D2Q9":
        C, om = lid_driven_cavity(m, model)
        s = C(lattice=m.LatticeD2Q9(PREC), omega=om(n[0]), nx=n[0], ny=n[1], nz=0, precision=PREC,
              print_info_rate=0)
    else:
        C, om = lid_driven_cavity_3d(m, model=model)
        lat = getattr(m, "Lattice" + lattice)(PREC)
        s = C(lattice=lat, omega=om(n[0]), nx=n[0], ny=n[1], nz=n[2], precision=PREC, print_info_rate=0)
    f = s.run(t_max)
    rho, u = s.update_macroscopic(f)
    return {"f": to_np(f), "rho": to_np(rho), "u": to_np(u)}


CASES = {
    "elast_plain_16x16": lambda m: elast_plain(m, 16, 16),
    "elast_plain_37x22": lambda m: elast_plain(m, 37, 22),
    "elast_periodic_mg3_32": lambda m: elast_periodic_mg(m),
    "elast_dirichlet_mg3": lambda m: elast_walled_mg(m, "dirichlet"),
    "elast_neumann_mg3": lambda m: elast_walled_mg(m, "neumann"),
    "elast_halfway": elast_halfway,
    "darcy_periodic": lambda m: darcy(m, "periodic"),
    "darcy_anti": lambda m: darcy(m, "anti"),
    "darcy_eq": lambda m: darcy(m, "eq"),
    "darcy_neumann": lambda m: darcy(m, "neumann"),
    "darcy_cell_omega": darcy_cell_omega,
    "biot_periodic_l1": lambda m: biot_periodic(m, 1),
    "biot_periodic_l2": lambda m: biot_periodic(m, 2),
    "biot_terzaghi_l3": biot_terzaghi,
    "mg_transfers": mg_transfers,
    "parameters_terzaghi": parameters_terzaghi,
    # the 'f64/f32' policy: FP64 arithmetic on FP32 storage (held to the FP32 bar)
    "elast_plain_16x16_f64f32": lambda m: elast_plain(m, 16, 16, prec="f64/f32"),
    "elast_dirichlet_mg3_f64f32": lambda m: elast_walled_mg(m, "dirichlet", prec="f64/f32"),
    "darcy_anti_f64f32": lambda m: darcy(m, "anti", prec="f64/f32"),
    "fluid_cavity_bgk_d2q9": lambda m: fluid_cavity(m, "bgk"),
    "fluid_cavity_kbc_d2q9": lambda m: fluid_cavity(m, "kbc"),
    "fluid_cavity_bgk_d3q19": lambda m: fluid_cavity(m, "bgk", "D3Q19", (10, 8, 12)),
    "fluid_cavity_bgk_d3q27": lambda m: fluid_cavity(m, "bgk", "D3Q27", (10, 8, 12)),
    "fluid_cavity_kbc_d3q27": lambda m: fluid_cavity(m, "kbc", "D3Q27", (10, 8, 12)),
}

# relative tolerance of each case (FP64 runs: 1e-12; FP32 storage: 1e-5)
TOLERANCE = {name: (1e-5 if name.endswith("_f64f32") else 1e-12) for name in CASES}
