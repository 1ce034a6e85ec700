"""Problem definitions shared by the oracle pins and the GPU parity tests.

Each builder takes a solver module namespace ``m`` (the oracle or the product)
exposing the reference's class names, so that the same hooks drive both.  The
manufactured solutions are the ones of the reference's examples
(``examples/elasticity/periodic.py:42-61``, ``examples/elasticity/dirichlet_MG.py``,
``examples/elasticity/neumann_MG.py``, ``examples/darcy/*.py``,
``examples/poroelasticity/periodic.py:51-149``, ``examples/poroelasticity/Terzaghi.py``).
"""
import numpy as np


def sum_function(nx, ny, kls, scale=lambda k, l: 1, shift=0.5, n_bc=0):
    """Sum of cos/sin products on cell centres, as ``sumFunction`` in the
    reference examples (``shift=-0.5, n_bc=2`` is the walled variant)."""
    def fun(f, g, k, l):
        return np.fromfunction(
            lambda x, y, d: scale(k, l) * f(k * np.pi * (x + shift) / (nx - n_bc))
            * g(l * np.pi * (y + shift) / (ny - n_bc)), (nx, ny, 1))
    val = np.zeros((nx, ny, 1))
    for j, fg in enumerate([(np.cos, np.cos), (np.cos, np.sin), (np.sin, np.cos), (np.sin, np.sin)]):
        for i in range(len(kls[j]) // 2):
            val += fun(*fg, kls[j][2 * i], kls[j][2 * i + 1])
    return val


def elastic_material(nu=0.8, E=0.11):
    """Plane-stress Lame parameters of the examples (``periodic.py:97-102``)."""
    return E * nu / (1 - nu ** 2), 0.5 * E / (1 + nu)


def periodic_elasticity_exact(nx, ny, lam, mu, shift=0.5, n_bc=0):
    eta = np.concatenate((sum_function(nx, ny, [[], [2, 2], [], []], lambda k, l: 9e-4, shift, n_bc),
                          sum_function(nx, ny, [[], [], [2, 2], []], lambda k, l: 7e-4, shift, n_bc)), axis=-1)
    sig = np.concatenate((
        sum_function(nx, ny, [[], [], [], [2, 2]], lambda k, l: np.pi * (-3.2e-3 * lam - 3.6e-3 * mu), shift, n_bc),
        sum_function(nx, ny, [[2, 2], [], [], []], lambda k, l: np.pi * 3.2e-3 * mu, shift, n_bc),
        sum_function(nx, ny, [[], [], [], [2, 2]], lambda k, l: np.pi * (-3.2e-3 * lam - 2.8e-3 * mu), shift, n_bc)),
        axis=-1)
    return eta, sig


def periodic_elasticity_force(nx, ny, lam, mu, shift=0.5, n_bc=0):
    eps = 1.0 / (nx - n_bc)
    return np.concatenate((
        sum_function(nx, ny, [[], [2, 2], [], []],
                     lambda k, l: eps ** 2 * np.pi ** 2 * (1.36e-2 * mu + 6.4e-3 * lam), shift, n_bc),
        sum_function(nx, ny, [[], [], [2, 2], []],
                     lambda k, l: eps ** 2 * np.pi ** 2 * (1.20e-2 * mu + 6.4e-3 * lam), shift, n_bc)), axis=-1)


def make_periodic_elasticity(m):
    """``examples/elasticity/periodic.py`` / ``periodic_MG.py`` (optionally with a
    random initial state so that short parity runs exercise every term)."""
    class PeriodicElasticity(m.LBMElasticity):
        init_seed = None

        def get_force(self):
            f = periodic_elasticity_force(self.nx, self.ny, self.lamda, self.mu)
            return self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.compute_dtype,
                                               init_val=f)

        def initialize_macroscopic_fields(self):
            if self.init_seed is None:
                return None, None
            rng = np.random.default_rng(self.init_seed)
            return (1e-3 * rng.standard_normal((self.nx, self.ny, 2)),
                    1e-3 * rng.standard_normal((self.nx, self.ny, 3)))

        def output_data(self, **kwargs):
            self.records = getattr(self, "records", [])
            self.records.append({k: (np.array(v) if v is not None and not np.isscalar(v) and k != "f_poststreaming"
                                     else v) for k, v in kwargs.items() if k != "f_poststreaming"})
    return PeriodicElasticity


def make_walled_elasticity(m, kind, mg_bcs=True):
    """``examples/elasticity/dirichlet_MG.py`` (kind='dirichlet', full-way
    bounce-back with wall displacement) and ``neumann_MG.py`` (kind='neumann',
    anti-bounce-back with traction)."""
    class Walled(m.LBMElasticity):
        def get_force(self):
            f = periodic_elasticity_force(self.nx, self.ny, self.lamda, self.mu, shift=-0.5, n_bc=2)
            f[0, ...] = 0.0
            f[1, ...] = 0.0
            f[:, 0, ...] = 0.0
            f[:, 1, ...] = 0.0
            return self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.compute_dtype,
                                               init_val=f)

        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            if kind == "dirichlet":
                eta_wall, _ = periodic_elasticity_exact(self.nx, self.ny, self.lamda, self.mu, -0.5, 2)
                Cls = m.ElasticityBounceBackFullway
                self.BCs.append(Cls(tuple(bb["left"].T), self.gridInfo, self.precisionPolicy, eta_wall[-1, ...]))
                self.BCs.append(Cls(tuple(bb["right"].T), self.gridInfo, self.precisionPolicy, eta_wall[0, ...]))
                self.BCs.append(Cls(tuple(bb["bottom"].T), self.gridInfo, self.precisionPolicy, eta_wall[:, -1, ...]))
                self.BCs.append(Cls(tuple(bb["top"].T), self.gridInfo, self.precisionPolicy, eta_wall[:, 0, ...]))
            else:
                _, sw = periodic_elasticity_exact(self.nx, self.ny, self.lamda, self.mu, -0.5, 2)

                def T_wall(n):
                    eps = 1.0 / (self.nx - 2)
                    return eps * np.stack((sw[..., 0] * n[0] + sw[..., 1] * n[1],
                                           sw[..., 1] * n[0] + sw[..., 2] * n[1]), axis=-1)
                Cls = m.ElasticityAntiBounceBack
                self.BCs.append(Cls(tuple(bb["left"].T), self.gridInfo, self.precisionPolicy, T_wall([-1, 0])[-1, 1:-1, ...]))
                self.BCs.append(Cls(tuple(bb["right"].T), self.gridInfo, self.precisionPolicy, T_wall([1, 0])[0, 1:-1, ...]))
                self.BCs.append(Cls(tuple(bb["bottom"].T), self.gridInfo, self.precisionPolicy, T_wall([0, -1])[1:-1, -1, ...]))
                self.BCs.append(Cls(tuple(bb["top"].T), self.gridInfo, self.precisionPolicy, T_wall([0, 1])[1:-1, 0, ...]))
            Cls = m.ElasticityBounceBackFullway if kind == "dirichlet" else m.ElasticityAntiBounceBack
            for level in range(1, self.levels):
                gi = self.grid_info(level)
                b = self.bounding_box_indices(level)
                self.BCs_MG[level] = [Cls(tuple(b[s].T), gi, self.precisionPolicy)
                                      for s in ("left", "right", "bottom", "top")]

        def output_data(self, **kwargs):
            self.records = getattr(self, "records", [])
            self.records.append({k: v for k, v in kwargs.items() if k != "f_poststreaming"})
    return Walled


DARCY_KLS = {"periodic": [[], [4, 4], [], [2, 2]], "anti": [[], [], [], [2, 4, 4, 2]],
             "eq": [[], [], [], [2, 4, 4, 2]], "neumann": [[2, 4, 4, 2], [], [], []]}


def make_darcy(m, kind):
    """``examples/darcy/{periodic,dirichlet,dirichlet_eq,neumann_bb}.py``."""
    walled = kind != "periodic"
    shift, n_bc = (-0.5, 2) if walled else (0.5, 0)

    class Darcy(m.AdvectionDiffusionReactionBGK):
        def __init__(self, **kwargs):
            self._kls = DARCY_KLS[kind]
            super().__init__(**kwargs)

        def get_source(self):
            K = (1.0 / self.omega - 0.5) / 3
            s = sum_function(self.nx, self.ny, self._kls,
                             lambda k, l: 0.5 * K * (k ** 2 + l ** 2) * np.pi ** 2 / (self.nx - n_bc) ** 2, shift, n_bc)
            if walled:
                s[(0, -1), :] = 0
                s[:, (0, -1)] = 0
            return self.distributed_array_init((self.nx, self.ny, 1), self.precisionPolicy.compute_dtype, init_val=s)

        def initialize_macroscopic_fields(self):
            p = sum_function(self.nx, self.ny, self._kls, shift=shift, n_bc=n_bc)
            p = self.distributed_array_init(p.shape, self.precisionPolicy.output_dtype, init_val=p)
            p = p - 0.5 * self.source
            vel = self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0)
            return p, vel

        def set_boundary_conditions(self):
            if not walled:
                return
            bb = self.boundingBoxIndices
            walls = np.concatenate((bb["left"], bb["right"], bb["top"], bb["bottom"]))
            if kind == "anti":
                self.BCs.append(m.ADR_AntiBounceBack(tuple(walls.T), self.gridInfo, self.precisionPolicy))
            elif kind == "eq":
                self.BCs.append(m.ADR_EquilibriumBC(tuple(walls.T), self.gridInfo, self.precisionPolicy, rho=0))
            else:
                self.BCs.append(m.ADR_Neumann_BounceBack(tuple(walls.T), self.gridInfo, self.precisionPolicy))

        def exact(self, timestep):
            Kt = (1.0 / self.omega - 0.5) / 3 * timestep / self.nx ** 2
            return sum_function(self.nx, self.ny, self._kls,
                                lambda k, l: 0.5 + 0.5 * np.exp(-Kt * (k ** 2 + l ** 2) * np.pi ** 2), shift, n_bc)

        def output_data(self, **kwargs):
            self.records = getattr(self, "records", [])
            self.records.append({"timestep": kwargs["timestep"], "rho": np.array(kwargs["rho"])})
    return Darcy


def corner_fixed_classes(m):
    """The corner-patched BC subclasses of ``examples/poroelasticity/Terzaghi.py:22-112``
    (they override ``get_missing_indices`` and mutate the boundary mask)."""
    def patched(base, table):
        class Patched(base):
            def get_missing_indices(self, boundaryMask):
                nbd = len(self.indices[0])
                imissing = np.vstack([np.arange(self.lattice.q, dtype='uint8')] * nbd)
                iknown = np.vstack([np.asarray(self.lattice.opp_indices)] * nbd)
                for i in range(nbd):
                    x, y = int(self.indices[0][i]), int(self.indices[1][i])
                    for (cx, cy), dirs in table(self.nx, self.ny).items():
                        if x == cx and y == cy:
                            for d in dirs:
                                boundaryMask[i, d] = False
                imissing[~boundaryMask] = 0
                iknown[~boundaryMask] = 0
                return imissing, iknown
        Patched.__name__ = base.__name__ + "Patched"
        return Patched

    adr_table = lambda nx, ny: {(1, 0): (1, 4), (1, ny - 1): (2, 8), (nx - 2, 0): (1, 7), (nx - 2, ny - 1): (2, 5)}
    el_table = lambda nx, ny: {(1, 0): (1, 5), (1, ny - 1): (3, 6), (nx - 2, 0): (1, 4), (nx - 2, ny - 1): (3, 7)}
    return (patched(m.ADR_Neumann_BounceBack, adr_table), patched(m.ADR_AntiBounceBack, adr_table),
            patched(m.ElasticityAntiBounceBack, el_table))


def make_periodic_biot(m, alpha=1.0):
    """``examples/poroelasticity/periodic.py:33-66`` (closed-form periodic Biot)."""
    class PD(m.AdvectionDiffusionReactionBGK):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((self.nx, self.ny, 1), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0))

    class PE(m.LBMElasticity):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((self.nx, self.ny, 3), self.precisionPolicy.output_dtype, init_val=0.0))

    class PP(m.LBMPoroelasticity):
        def __init__(self, **kwargs):
            super().__init__(PE, PD, **kwargs)

        def get_elastic_force(self, timestep):
            K = (1.0 / self.darcy.omega - 0.5) / 3
            el = self.elasticity
            tf = 1 - np.exp(-8 * np.pi ** 2 * K * timestep / el.nx ** 2)
            force = np.concatenate((sum_function(el.nx, el.ny, [[], [2, 2], [], []],
                                                 lambda k, l: self.epsilon ** 2 * tf * np.pi ** 2 * 8 * el.mu),
                                    np.zeros((el.nx, el.ny, 1))), axis=-1)
            return el.distributed_array_init((el.nx, el.ny, 2), el.precisionPolicy.compute_dtype, init_val=force)

        def get_darcy_source(self, timestep):
            K = (1.0 / self.darcy.omega - 0.5) / 3
            el, da = self.elasticity, self.darcy
            tf = np.exp(-8 * np.pi ** 2 * K * timestep / el.nx ** 2)
            factor = -np.pi ** 3 * K / da.nx ** 2 * (128 * self.alpha * tf + (128 * el.lamda + 240 * el.mu) / self.alpha)
            s = sum_function(da.nx, da.ny, [[], [], [], [2, 2]], lambda k, l: factor)
            return da.distributed_array_init((da.nx, da.ny, 1), da.precisionPolicy.compute_dtype, init_val=s)

        def output_data(self, **kwargs):
            self.records = getattr(self, "records", [])
            self.records.append({k: np.array(v) for k, v in kwargs.items()
                                 if k in ("timestep", "eta", "sigma", "pressure", "pressure_grad", "dt_div_eta")})
    return PP


def periodic_biot_exact(nx, ny, lam, mu, alpha, K, timestep):
    """``examples/poroelasticity/periodic.py:92-149``."""
    tf = 1 - np.exp(-8 * np.pi ** 2 * K * timestep / nx ** 2)
    eta = np.concatenate((sum_function(nx, ny, [[], [2, 2], [], []], lambda k, l: 4.5 * tf),
                          sum_function(nx, ny, [[], [], [2, 2], []], lambda k, l: 3.5 * tf)), axis=-1)
    p = sum_function(nx, ny, [[], [], [], [2, 2]], lambda k, l: -np.pi / alpha * tf * (16 * lam + 30 * mu))
    return eta, p


def make_terzaghi(m, force_value=-1.0, ny=4):
    """Quasi-1D Terzaghi consolidation set-up (``examples/poroelasticity/Terzaghi.py:115-154``):
    Darcy no-flux left / drained right, elasticity clamped left / loaded right,
    corner-patched BCs, ``MG_BCs`` left/right."""
    ADR_BB, ADR_AntiBB, ElasticityAntiBB = corner_fixed_classes(m)

    class TD(m.AdvectionDiffusionReactionBGK):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((self.nx, self.ny, 1), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0))

        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            self.BCs.append(ADR_BB(tuple(bb["left"].T), self.gridInfo, self.precisionPolicy))
            self.BCs.append(ADR_AntiBB(tuple(bb["right"].T), self.gridInfo, self.precisionPolicy))

    class TE(m.LBMElasticity):
        def initialize_macroscopic_fields(self):
            return (self.distributed_array_init((self.nx, self.ny, 2), self.precisionPolicy.output_dtype, init_val=0.0),
                    self.distributed_array_init((self.nx, self.ny, 3), self.precisionPolicy.output_dtype, init_val=0.0))

        def set_boundary_conditions(self):
            bb = self.boundingBoxIndices
            self.BCs.append(m.ElasticityBounceBackFullway(tuple(bb["left"].T), self.gridInfo, self.precisionPolicy))
            force = np.stack((np.full((self.ny,), force_value), np.zeros((self.ny,))), axis=-1)
            self.BCs.append(ElasticityAntiBB(tuple(bb["right"].T), self.gridInfo, self.precisionPolicy, force))
            for level in range(1, self.levels):
                gi = self.grid_info(level)
                b = self.bounding_box_indices(level)
                self.BCs_MG[level] = [m.ElasticityBounceBackFullway(tuple(b["left"].T), gi, self.precisionPolicy),
                                      ElasticityAntiBB(tuple(b["right"].T), gi, self.precisionPolicy)]

    class TP(m.LBMPoroelasticity):
        def __init__(self, **kwargs):
            super().__init__(TE, TD, **kwargs)

        def output_data(self, **kwargs):
            self.records = getattr(self, "records", [])
            self.records.append({k: np.array(v) for k, v in kwargs.items()
                                 if k in ("timestep", "eta", "sigma", "pressure", "pressure_grad", "dt_div_eta")})
    return TP


def make_cavity(m, model="bgk", u_wall=0.1, Re=100.0):
    """``examples/performance/MLUPS2d.py`` (the benchmark workload of the same
    name): returns the cavity class and ``omega(n)``."""
    from xlb_biot_b200.workloads import lid_driven_cavity
    return lid_driven_cavity(m, model, u_wall, Re)


def make_shear_wave(m, model="bgk", amp=0.02):
    """Periodic decaying shear wave u_x(y) = amp sin(2 pi (y + 1/2) / ny) at
    rho = 1: the incompressible solution decays as exp(-nu k^2 t) with
    nu = (1 / omega - 1/2) / 3 and k = 2 pi / ny."""
    base = m.BGKSim if model == "bgk" else m.KBCSim

    class ShearWave(base):
        def initialize_macroscopic_fields(self):
            y = (np.arange(self.ny) + 0.5) / self.ny
            u = np.zeros((self.nx, self.ny, 2))
            u[..., 0] = amp * np.sin(2 * np.pi * y)[None, :]
            rho = np.ones((self.nx, self.ny, 1))
            dt = self.precisionPolicy.compute_dtype
            return rho.astype(dt), u.astype(dt)
    return ShearWave
