"""D2Q8 linear-elasticity LBM with geometric multigrid on B200.

Drop-in for ``src/elasticity.py`` of the reference: the class
``LBMElasticity`` keeps the reference's constructor keywords, validation,
hooks (``set_boundary_conditions``, ``get_force``,
``initialize_macroscopic_fields``, ``output_data``) and public methods; the
three elasticity boundary conditions keep their signatures.  Every sweep runs
in the fused CUDA kernel ``xlbb_elast_sweep`` (collide + BCs + stream, with the
multigrid smoother / residual algebra folded in); macroscopic fields, the
equilibrium and the multigrid transfers have their own kernels.
"""
import time

import numpy as np
import torch

from . import _lib
from ._common import (gathered, iterate_to_tolerance, make_policy, print_parameters, require_finite,
                      set_precisions, storage_and_sweep_dtypes)
from .bc_compile import apply_rules_device, compile_rules
from .boundary_conditions import (BoundaryCondition, _at_add, _at_set, _take, grid_mask, solid_halo_voxels)
from .fields import Layout, torch_dtype


def coarsen_material(a, mg_bcs):
    """Material field of the next coarser multigrid level (torch, differentiable).

    Extension without a reference counterpart (the reference has uniform
    Lame parameters).  Interior cells: mean of the 2 x 2 fine block (the
    block the restriction sums); boundary rows / columns kept by ``MG_BCs``:
    mean of the fine pair along the boundary; corners: copied."""
    l, r, b, t = (int(mg_bcs[k]) for k in ("left", "right", "bottom", "top"))
    nx, ny = a.shape
    inner = a[l:nx - r, b:ny - t]
    c = 0.25 * (inner[0::2, 0::2] + inner[1::2, 0::2] + inner[0::2, 1::2] + inner[1::2, 1::2])
    if b:
        c = torch.cat([(0.5 * (a[l:nx - r, 0][0::2] + a[l:nx - r, 0][1::2]))[:, None], c], 1)
    if t:
        c = torch.cat([c, (0.5 * (a[l:nx - r, ny - 1][0::2] + a[l:nx - r, ny - 1][1::2]))[:, None]], 1)

    def column(x):
        mid = 0.5 * (a[x, b:ny - t][0::2] + a[x, b:ny - t][1::2])
        parts = ([a[x, 0:1]] if b else []) + [mid] + ([a[x, ny - 1:ny]] if t else [])
        return torch.cat(parts)[None, :]
    if l:
        c = torch.cat([column(0), c], 0)
    if r:
        c = torch.cat([c, column(nx - 1)], 0)
    return c


def material_hierarchy(lam, mu, mg_bcs, levels):
    """Per-level (lambda, mu) fields: level 0 as given, each coarser level by
    ``coarsen_material``."""
    out = [(lam, mu)]
    for _ in range(1, levels):
        lam, mu = coarsen_material(lam, mg_bcs), coarsen_material(mu, mg_bcs)
        out.append((lam, mu))
    return out


class LBMElasticity:
    """``src/elasticity.py:30-1501``."""

    def __init__(self, **kwargs):
        self._init_kwargs = dict(kwargs)       # an FP64 twin is built from them (refine.py)
        # the poroelastic coupling force fused into the smoothing sweeps (same values)
        self._fused_coupling = bool(kwargs.get("fused_coupling", True))
        self.lamda = kwargs.get("lambda")
        self.mu = kwargs.get("mu")
        self.nx = kwargs.get("nx")
        self.ny = kwargs.get("ny")
        self.nz = kwargs.get("nz")
        self.mg_BCs = kwargs.get("MG_BCs", {})
        self.levels = kwargs.get("MG_levels", 1)
        self.gamma = kwargs.get("MG_relaxation", 0.75)
        self.k_smooth = kwargs.get("MG_n_smoothing", 2)
        self.precision = kwargs.get("precision")
        self.precisionPolicy = make_policy(self.precision)
        self.lattice = kwargs.get("lattice")
        self.downsamplingFactor = kwargs.get("downsampling_factor", 1)
        self.printInfoRate = kwargs.get("print_info_rate", 100)
        self.ioRate = kwargs.get("io_rate", 0)
        self.returnFpost = kwargs.get("return_fpost", False)
        self.computeMLUPS = kwargs.get("compute_MLUPS", False)
        self.nDevices = 1
        self.backend = "cuda"
        if self.computeMLUPS:
            self.ioRate = 0
            self.printInfoRate = 0
        _lib.require_cuda()
        _lib.lib()
        self.c, self.q, self.w, self.dim = self.lattice.c, self.lattice.q, self.lattice.w, self.lattice.d
        self._create_transfer_matrices()
        self.show_simulation_parameters()
        self.gridInfo = {"nx": self.nx, "ny": self.ny, "nz": self.nz, "dim": self.lattice.d, "lattice": self.lattice}
        self.sharding = None
        # storage type of the fields; under 'f64/f32' every sweep computes in
        # FP64 (dtype code XLBB_F32_ACC64, FP64 rule constants) on FP32 fields
        self._dtype, self._acc64_all = storage_and_sweep_dtypes(self.precisionPolicy)
        self._dcode = _lib.dtype_code(self._dtype)
        # Extension: ``coarsest_precision="f64"`` runs the coarsest multigrid level
        # in FP64 under FP32 levels (transfers convert in the kernels).
        self._level_dtypes = [self._dtype] * self.levels
        if kwargs.get("coarsest_precision") == "f64" and self.levels > 1:
            self._level_dtypes[-1] = torch.float64
        self._layouts = [Layout(*self.grid_size(l), self._level_dtypes[l]) for l in range(self.levels)]
        # Extension: ``residual_precision="f64"`` computes the level-0 residual sweep
        # of an FP32 multigrid solve in FP64 arithmetic (FP32 storage): the coarse
        # corrections then see the residual of the stored state without FP32
        # rounding noise, which otherwise limits the solution's accuracy.
        self._res64 = (kwargs.get("residual_precision") == "f64" and self.levels > 1
                       and self._level_dtypes[0] == torch.float32)
        self.boundingBoxIndices = self.bounding_box_indices()
        self._create_boundary_data()
        force = self.get_force()
        self.force = self._layouts[0].field(force, 2) if force is not None else None
        self._mat = _lib.ElastMaterial(float(self.lamda), float(self.mu), None, None)
        self._mats = [self._mat] * self.levels
        # Extension: per-cell Lame fields (``lambda_field``, ``mu_field``, shape
        # (nx, ny) or (nx, ny, 1)); coarse levels use ``coarsen_material``.
        self._lam_fields = self._mu_fields = None
        lf, mf = kwargs.get("lambda_field"), kwargs.get("mu_field")
        if (lf is None) != (mf is None):
            raise ValueError("lambda_field and mu_field go together")
        if lf is not None:
            self.set_material_fields(lf, mf)
        self._div_scale = -1.5 / (3 * (self.lamda + self.mu) + 1)
        self._partials = torch.empty(0, dtype=torch.float64, device=self._layouts[0].device)
        self._n_partials = 0
        self._scalar = torch.empty(1, dtype=torch.float64, device=self._layouts[0].device)

    # ------------------------------------------------------------------ validation
    @property
    def lattice(self):
        return self._lattice

    @lattice.setter
    def lattice(self, value):
        if value is None:
            raise ValueError("Lattice type must be provided.")
        if self.nz == 0 and value.name not in ["D2Q8"]:
            raise ValueError("For 2D simulations, lattice type must be LatticeD2Q8.")
        if self.nz != 0:
            raise ValueError("3D simulations are not supported.")
        self._lattice = value

    @property
    def lamda(self):
        return self._lamda

    @lamda.setter
    def lamda(self, value):
        if value is None:
            raise ValueError("lambda must be provided")
        if not isinstance(value, float):
            raise TypeError("lambda must be a float")
        self._lamda = value

    @property
    def mu(self):
        return self._mu

    @mu.setter
    def mu(self, value):
        if value is None:
            raise ValueError("mu must be provided")
        if not isinstance(value, float):
            raise TypeError("mu must be a float")
        self._mu = value

    @property
    def levels(self):
        return self._levels

    @levels.setter
    def levels(self, value):
        if value is None:
            raise ValueError("levels must be provided")
        if not isinstance(value, int) or value <= 0:
            raise TypeError("levels must be a positive int")
        den = 2 ** (value - 1)
        m = self.mg_BCs
        if ((self.nx - int(m["left"]) - int(m["right"])) % den != 0
                or (self.ny - int(m["bottom"]) - int(m["top"])) % den != 0
                or (self.nz - int(m["front"]) - int(m["back"])) % den != 0):
            raise ValueError("nx,ny,nz (-BCs) must be divisible by 2**(levels-1)")
        self._levels = value

    @property
    def gamma(self):
        return self._gamma

    @gamma.setter
    def gamma(self, value):
        if value is None:
            raise ValueError("gamma must be provided")
        if not isinstance(value, float):
            raise TypeError("gamma must be a float")
        if value < 0.0 or value > 1.0:
            raise ValueError("gamma must be between 0 and 1")
        self._gamma = value

    @property
    def k_smooth(self):
        return self._k_smooth

    @k_smooth.setter
    def k_smooth(self, value):
        if value is None:
            raise ValueError("k_smooth must be provided")
        if not isinstance(value, int):
            raise TypeError("k_smooth must be an integer")
        if value < 1:
            raise ValueError("k_smooth must be positive")
        self._k_smooth = value

    @property
    def mg_BCs(self):
        return self._mg_BCs

    @mg_BCs.setter
    def mg_BCs(self, value):
        if not isinstance(value, dict):
            raise TypeError("mg_BCs must be a dictionary")
        for key, bc in value.items():
            if key not in ["left", "right", "bottom", "top", "front", "back"]:
                raise ValueError(f"Invalid key '{key}' in mg_BCs. Valid keys are 'left', 'right', 'bottom', "
                                 "'top', 'front', 'back'.")
            if not isinstance(bc, bool):
                raise TypeError("All values in mg_BCs must be boolean values")
        self._mg_BCs = {"left": False, "right": False, "bottom": False, "top": False, "front": False,
                        "back": False}
        self._mg_BCs.update(value)

    def _int_prop(name, label):
        def getter(self):
            return getattr(self, "_" + name)

        def setter(self, value):
            if value is None and label in ("nx", "ny", "nz"):
                raise ValueError(f"{label} must be provided")
            if not isinstance(value, int) or isinstance(value, bool):
                raise TypeError(f"{label} must be an integer")
            setattr(self, "_" + name, value)
        return property(getter, setter)

    nx = _int_prop("nx", "nx")
    ny = _int_prop("ny", "ny")
    nz = _int_prop("nz", "nz")
    downsamplingFactor = _int_prop("downsamplingFactor", "downsamplingFactor")
    printInfoRate = _int_prop("printInfoRate", "printInfoRate")
    ioRate = _int_prop("ioRate", "ioRate")
    nDevices = _int_prop("nDevices", "nDevices")

    def _bool_prop(name, label):
        def getter(self):
            return getattr(self, "_" + name)

        def setter(self, value):
            if not isinstance(value, bool):
                raise TypeError(f"{label} must be a boolean")
            setattr(self, "_" + name, value)
        return property(getter, setter)

    returnFpost = _bool_prop("returnFpost", "returnFpost")
    computeMLUPS = _bool_prop("computeMLUPS", "computeMLUPS")
    del _int_prop, _bool_prop

    @property
    def precision(self):
        return self._precision

    @precision.setter
    def precision(self, value):
        if not isinstance(value, str):
            raise TypeError("precision must be a string")
        self._precision = value

    def show_simulation_parameters(self):
        attrs = ['lamda', 'mu', 'nx', 'ny', 'nz', 'dim', 'levels', 'gamma', 'k_smooth', 'precision', 'lattice',
                 'downsamplingFactor', 'printInfoRate', 'ioRate', 'computeMLUPS', 'backend', 'nDevices']
        names = {'lamda': 'Lambda', 'mu': 'Mu', 'nx': 'Grid Points in X', 'ny': 'Grid Points in Y',
                 'nz': 'Grid Points in Z', 'dim': 'Dimensionality', 'levels': 'Multigrid levels',
                 'gamma': 'Multigrid relaxation factor', 'k_smooth': 'Multigrid smoothing steps',
                 'precision': 'Precision Policy', 'lattice': 'Lattice Type',
                 'downsamplingFactor': 'Downsampling Factor', 'printInfoRate': 'Print Info Rate',
                 'ioRate': 'I/O Rate', 'computeMLUPS': 'Compute MLUPS', 'backend': 'Backend',
                 'nDevices': 'Number of Devices'}
        print_parameters(self, attrs, names)

    # ------------------------------------------------------------------ set-up
    def set_precisions(self, precision):
        return set_precisions(precision)

    def _create_transfer_matrices(self):
        """``:805-848`` (kept for API parity; the kernels hard-code the same matrices)."""
        g = 1.0 / (12.0 * (self.lamda + self.mu) - 4.0)
        if abs(g) > 100:
            print("Warning: scaling value is too large. Reset last moment to default. Boundary conditions may fail.")
            g = 0.0
        dt = self.precisionPolicy.compute_dtype
        self.f_to_m = np.array([[1, 0, -1, 0, 1, -1, -1, 1], [0, 1, 0, -1, 1, 1, -1, -1],
                                [1, 1, 1, 1, 2, 2, 2, 2], [1, -1, 1, -1, 0, 0, 0, 0],
                                [0, 0, 0, 0, 1, -1, 1, -1]], dtype=dt).T
        h, n = 0.25 + 0.5 * g, -0.25 * g
        self.m_to_f = np.array([[0.5, 0, h, 0.25, 0, -0.5, 0], [0, 0.5, h, -0.25, 0, 0, -0.5],
                                [-0.5, 0, h, 0.25, 0, 0.5, 0], [0, -0.5, h, -0.25, 0, 0, 0.5],
                                [0, 0, n, 0, 0.25, 0.25, 0.25], [0, 0, n, 0, -0.25, -0.25, 0.25],
                                [0, 0, n, 0, 0.25, -0.25, -0.25], [0, 0, n, 0, -0.25, 0.25, -0.25]], dtype=dt).T

    def grid_size(self, level=0):
        """``:501-529``."""
        if level == 0:
            return self.nx, self.ny
        nxb = int(self.mg_BCs["left"]) + int(self.mg_BCs["right"])
        nyb = int(self.mg_BCs["bottom"]) + int(self.mg_BCs["top"])
        return (self.nx - nxb) // 2 ** level + nxb, (self.ny - nyb) // 2 ** level + nyb

    def grid_info(self, level=0):
        nx, ny = self.grid_size(level)
        return {"nx": nx, "ny": ny, "nz": self.nz, "dim": self.lattice.d, "lattice": self.lattice}

    def bounding_box_indices(self, level=0):
        """``:563-589``."""
        nx, ny = self.grid_size(level)
        return {"bottom": np.array([[i, 0] for i in range(nx)], dtype=int),
                "top": np.array([[i, ny - 1] for i in range(nx)], dtype=int),
                "left": np.array([[0, i] for i in range(ny)], dtype=int),
                "right": np.array([[nx - 1, i] for i in range(ny)], dtype=int)}

    def create_grid_mask(self, solid_halo_voxels, level=0):
        nx, ny = self.grid_size(level)
        return grid_mask(nx, ny, self.lattice, solid_halo_voxels)

    def _create_boundary_data(self):
        """``:396-436``, then compilation of each level's BC list into kernel rules."""
        self.BCs = []
        self.BCs_MG = {level: [] for level in range(1, self.levels)}
        self.set_boundary_conditions()
        t0 = time.time()
        for level in range(self.levels):
            bcs = self.BCs if level == 0 else self.BCs_MG[level]
            gm = self.create_grid_mask(solid_halo_voxels(bcs), level)
            for bc in bcs:
                assert bc.implementationStep in ['PostStreaming', 'PostCollision']
                bc.create_local_mask_and_normal_arrays(gm)
        self._compile_rules()
        print("Time to create the grid masks and boundary rules:", time.time() - t0)

    def _compile_rules(self):
        self._rules = []
        for level in range(self.levels):
            bcs = self.BCs if level == 0 else self.BCs_MG[level]
            L = self._layouts[level]
            rd = self._sweep_rule_dtype(L)
            pc = compile_rules(bcs, L.nx, L.ny, 8, rd, L.device, step="PostCollision")
            ps = compile_rules(bcs, L.nx, L.ny, 8, rd, L.device, step="PostStreaming")
            self._rules.append((pc, ps))
        if self._res64:      # FP64 rule constants of the FP64-arithmetic residual sweep
            L = self._layouts[0]
            self._rules_acc64 = (compile_rules(self.BCs, L.nx, L.ny, 8, torch.float64, L.device, step="PostCollision"),
                                 compile_rules(self.BCs, L.nx, L.ny, 8, torch.float64, L.device, step="PostStreaming"))

    def _sweep_acc64(self, L):
        """Whether sweeps on a level of layout L compute in FP64 on FP32 storage."""
        return self._acc64_all and L.dtype == torch.float32

    def _sweep_rule_dtype(self, L):
        return torch.float64 if self._sweep_acc64(L) else L.dtype

    def distributed_array_init(self, shape, type, init_val=0, sharding=None):
        """A device field of ``shape`` filled with ``init_val`` (``:438-458``)."""
        dt = torch_dtype(type)
        if len(shape) == 3:
            return Layout(shape[0], shape[1], dt).field(init_val, shape[2])
        x = torch.as_tensor(np.asarray(init_val) if not isinstance(init_val, torch.Tensor) else init_val)
        return torch.broadcast_to(x.to(device="cuda", dtype=dt), shape).clone()

    # ------------------------------------------------------------------ hooks
    def initialize_macroscopic_fields(self):
        print("WARNING: Default initial conditions assumed: displacement = 0, stress = 0")
        print("         To set explicit initial displacement and stress, use self.initialize_macroscopic_fields.")
        return None, None

    def output_data(self, **kwargs):
        pass

    def set_boundary_conditions(self):
        pass

    def get_force(self):
        pass

    # ------------------------------------------------------------------ material fields
    def set_material_fields(self, lam_field, mu_field):
        """Per-cell Lame fields on every level (written in place, so CUDA graphs
        captured earlier see the new values)."""
        dev = self._layouts[0].device

        def as2d(x):
            t = torch.as_tensor(x.detach() if isinstance(x, torch.Tensor) else np.asarray(x),
                                dtype=torch.float64, device=dev)
            return t.reshape(self.nx, self.ny)
        hier = material_hierarchy(as2d(lam_field), as2d(mu_field), self.mg_BCs, self.levels)
        if self._lam_fields is None:
            self._lam_fields = [self._L(l).empty(1) for l in range(self.levels)]
            self._mu_fields = [self._L(l).empty(1) for l in range(self.levels)]
        for l, (lam, mu) in enumerate(hier):
            self._lam_fields[l].copy_(lam[..., None])
            self._mu_fields[l].copy_(mu[..., None])
        self._mats = [_lib.ElastMaterial(float(self.lamda), float(self.mu), self._lam_fields[l].data_ptr(),
                                         self._mu_fields[l].data_ptr()) for l in range(self.levels)]

    def material_fields(self, level=0):
        """(lambda, mu) fields of ``level`` (None if uniform)."""
        if self._lam_fields is None:
            return None, None
        return self._lam_fields[level], self._mu_fields[level]

    # ------------------------------------------------------------------ fields
    def _L(self, level=0):
        return self._layouts[level]

    def _f(self, f, level=0):
        return self._L(level).field(f, 8)

    def assign_fields_sharded(self):
        """``:647-679``."""
        eta0, sigma0 = self.initialize_macroscopic_fields()
        if eta0 is None or sigma0 is None:
            return self._L().zeros(8)
        return self.initialize_populations(eta0, sigma0)

    def initialize_populations(self, eta0, sigma0):
        return self.equilibrium(eta0, sigma0)

    def equilibrium(self, eta, sigma, cast_output=True, external_force=None):
        """``:909-957`` (kernel ``xlbb_elast_equilibrium``)."""
        L = self._L()
        out = L.empty(8)
        fe = L.field(external_force, 2)
        # device copies must stay referenced until the asynchronous launch is enqueued:
        # a freed temporary's block is handed to the next allocation on the stream
        eta_d, sigma_d = L.field(eta, 2), L.field(sigma, 3)
        _lib.check(_lib.lib().xlbb_elast_equilibrium(
            self._dcode, L.grid(), self._mats[0], _lib.ptr(eta_d), _lib.ptr(sigma_d),
            _lib.ptr(self.force), _lib.ptr(fe), _lib.ptr(out), _lib.stream_ptr()), "xlbb_elast_equilibrium")
        return out

    def update_macroscopic(self, f, external_force=None):
        """``:1002-1038`` (kernel ``xlbb_elast_moments``)."""
        L = self._L()
        f = self._f(f)
        eta, sigma = L.empty(2), L.empty(3)
        fe = L.field(external_force, 2)
        _lib.check(_lib.lib().xlbb_elast_moments(
            self._dcode, L.grid(), self._mats[0], _lib.ptr(f), _lib.ptr(self.force), _lib.ptr(fe),
            _lib.ptr(eta), _lib.ptr(sigma), None, 0.0, _lib.stream_ptr()), "xlbb_elast_moments")
        return eta, sigma

    def update_divergence(self, f, level=None):
        """``:1040-1058`` (kernel ``xlbb_elast_moments``)."""
        if level is None:
            level = self._level_of(f)
        L = self._L(level)
        f = self._f(f, level)
        div = L.empty(1)
        _lib.check(_lib.lib().xlbb_elast_moments(
            _lib.dtype_code(L.dtype), L.grid(), self._mats[level], _lib.ptr(f), None, None, None, None, _lib.ptr(div),
            self._div_scale, _lib.stream_ptr()), "xlbb_elast_moments")
        return div

    def coupling_force(self, f, level, darcy, scale, base=None):
        """``base + darcy.gradient(self.update_divergence(f, level), scale)`` on
        multigrid level ``level`` in that level's precision, in one kernel
        (``xlbb_elast_divgrad``: the same values bit for bit).  The poroelastic
        coupling force of ``src/poroelasticity.py:324``."""
        L = self._L(level)
        f = self._f(f, level)
        base = L.field(base, 2)
        out = L.empty(2)
        rules = darcy.gradient_rules(L.nx, L.ny, L.dtype)
        _lib.check(_lib.lib().xlbb_elast_divgrad(
            _lib.dtype_code(L.dtype), L.grid(), self._mats[level], self._div_scale, _lib.ptr(f), float(scale),
            rules.struct(), _lib.ptr(base), _lib.ptr(out), _lib.stream_ptr()), "xlbb_elast_divgrad")
        return out

    def _level_of(self, f):
        shape = tuple(f.shape[:2])
        for level in range(self.levels):
            if shape == self.grid_size(level):
                return level
        raise ValueError(f"array of shape {tuple(f.shape)} matches no multigrid level")

    # ------------------------------------------------------------------ reference-compatible pieces
    def collision(self, f, external_force, use_force=True):
        """``:959-1000``: the collision alone (API compatibility; the time loop
        uses the fused sweep).  Computed on the device with tensor algebra."""
        level = self._level_of(f)
        fd = self._f(f, level).permute(0, 1, 2)
        F = None
        if use_force and self.force is not None and external_force is not None:
            F = self.force + self._L(level).field(external_force, 2)
        elif external_force is not None:
            F = self._L(level).field(external_force, 2)
        elif use_force and self.force is not None:
            F = self.force
        f2m = torch.as_tensor(self.f_to_m, device=fd.device, dtype=fd.dtype)
        m2f = torch.as_tensor(self.m_to_f, device=fd.device, dtype=fd.dtype)
        m = fd @ f2m
        lam_f, mu_f = self.material_fields(level)
        if lam_f is None:
            lam, mu = self.lamda, self.mu
        else:
            lam, mu = lam_f.to(fd.dtype), mu_f.to(fd.dtype)
        cs = (3 * (lam + mu) - 1) / (3 * (lam + mu) + 1)
        cd = (6 * mu - 1) / (6 * mu + 1)
        if F is not None:
            m = torch.cat([m[..., 0:2] + F, m[..., 2:3] * cs, m[..., 3:5] * cd, m[..., 0:2] / 3.0 + F / 6.0], -1)
        else:
            m = torch.cat([m[..., 0:2], m[..., 2:3] * cs, m[..., 3:5] * cd, m[..., 0:2] / 3.0], -1)
        if lam_f is None:
            return self._L(level).field(m @ m2f, 8)
        # per-cell m_to_f: only the ms row (h for the axis, n for the diagonal directions) varies
        g = 1.0 / (12.0 * (lam + mu) - 4.0)
        g = torch.where(g.abs() > 100, torch.zeros_like(g), g)
        hn = torch.cat([(0.25 + 0.5 * g).expand(*g.shape[:2], 4), (-0.25 * g).expand(*g.shape[:2], 4)], -1)
        m2f0 = m2f.clone()
        m2f0[2, :] = 0
        return self._L(level).field(m @ m2f0 + m[..., 2:3] * hn, 8)

    def streaming(self, f):
        """Periodic pull streaming (``:738-803``; API compatibility)."""
        out = torch.empty_like(f)
        for i in range(self.q):
            out[..., i] = torch.roll(f[..., i], (int(self.c[0, i]), int(self.c[1, i])), dims=(0, 1))
        return out

    def apply_bc(self, fout, fin, timestep, implementation_step, level=0):
        """``:1061-1091`` (API compatibility) with the compiled rules."""
        pc, ps = self._rules[level]
        return apply_rules_device(pc if implementation_step == "PostCollision" else ps, fout, fin)

    def apply_mg_bc(self, fout, fin, timestep, implementation_step, level):
        return self.apply_bc(fout, fin, timestep, implementation_step, level)

    def _interior(self, shape):
        return (slice(int(self.mg_BCs["left"]), shape[0] - int(self.mg_BCs["right"])),
                slice(int(self.mg_BCs["bottom"]), shape[1] - int(self.mg_BCs["top"])))

    def _box(self, level):
        nx, ny = self.grid_size(level)
        m = self.mg_BCs
        return int(m["left"]), nx - int(m["right"]), int(m["bottom"]), ny - int(m["top"])

    def substract_residual(self, f, residual):
        """``:1314-1344``."""
        if residual is None:
            return f
        level = self._level_of(f)
        out = self._f(f, level).clone()
        out[self._interior(out.shape)] -= residual.to(out.dtype)
        return out

    def _restrict(self, f):
        """``:850-865``: returns the 2x2 block sums of the interior (reference shape)."""
        level = self._level_of(f)
        rc = self._restrict_full(self._f(f, level), level)
        return rc[self._interior(rc.shape)]

    def _prolong(self, f):
        """``:878-894``: injection of the coarse interior to twice its size."""
        if not isinstance(f, torch.Tensor):
            f = torch.as_tensor(np.asarray(f), device=self._L(0).device)
        s = f[self._interior(f.shape)]
        return s.repeat_interleave(2, dim=0).repeat_interleave(2, dim=1)

    # ------------------------------------------------------------------ kernels
    def _sweep(self, f, level, a=0.0, b=1.0, resid=None, fext=None, out=None, sumsq=False, div_out=None,
               sumsq_diff=False, acc64=False, query=False, homogeneous=False, coupling=None):
        """One fused sweep on ``level``; ``acc64``: FP64 arithmetic on the FP32
        level-0 fields (``residual_precision="f64"``).  ``query``: launch
        nothing, return the pipeline the library would run (diagnostic).
        ``homogeneous``: the linear part of the sweep (no static force,
        boundary constants zero; a refinement step's correction)."""
        L = self._L(level)
        out = L.empty(8) if out is None else out
        if fext is not None and not L.conforms(fext, 2):
            fext = L.field(fext, 2)      # e.g. a coupling force computed in another precision
        acc64_all = self._sweep_acc64(L)
        code = _lib.XLBB_F32_ACC64 if (acc64 or acc64_all) else _lib.dtype_code(L.dtype)
        if sumsq:
            # a buffer for the largest launch shape; the reduction reads the
            # partials of the launch this sweep takes
            n_max = _lib.check(_lib.lib().xlbb_elast_sweep_ctas(code, L.grid()), "xlbb_elast_sweep_ctas")
            if self._partials.numel() < n_max:
                self._partials = torch.empty(n_max, dtype=torch.float64, device=L.device)
        pc, ps = self._rules_acc64 if (acc64 and not acc64_all) else self._rules[level]
        force = self.force
        if homogeneous:
            pc, ps = self._homogeneous_rules(level)
            force = None
        bx0, bx1, by0, by1 = self._box(level)
        s = _lib.ElastSweep(f.data_ptr(), out.data_ptr(), force.data_ptr() if force is not None else None,
                            1 if level == 0 and force is not None else 0, fext.data_ptr() if fext is not None else None,
                            resid.data_ptr() if resid is not None else None, float(a), float(b),
                            pc.struct(), ps.struct(), self._partials.data_ptr() if sumsq else None,
                            bx0, bx1, by0, by1, div_out.data_ptr() if div_out is not None else None,
                            1 if sumsq_diff else 0)
        if query:
            return _lib.check(_lib.lib().xlbb_elast_sweep_pipeline(code, L.grid(), self._mats[level], s),
                              "xlbb_elast_sweep_pipeline")
        if coupling is not None:         # fext is the coupling force's base: the force is computed in-kernel
            rules = coupling.darcy.gradient_rules(L.nx, L.ny, L.dtype)
            st = _lib.lib().xlbb_elast_sweep_divgrad(code, L.grid(), self._mats[level], s, self._div_scale,
                                                     float(coupling.scale), rules.struct(), _lib.stream_ptr())
            if st == _lib.XLBB_EUNSUPPORTED:
                return None
            _lib.check(st, "xlbb_elast_sweep_divgrad")
            return out
        if sumsq:
            self._n_partials = _lib.check(_lib.lib().xlbb_elast_sweep_partials(code, L.grid(), self._mats[level], s),
                                          "xlbb_elast_sweep_partials")
        _lib.check(_lib.lib().xlbb_elast_sweep(code, L.grid(), self._mats[level], s, _lib.stream_ptr()),
                   "xlbb_elast_sweep")
        return out

    def _homogeneous_rules(self, level):
        cache = self.__dict__.setdefault("_hom_rules", {})
        if level not in cache:
            from .refine import homogeneous_rules
            L = self._L(level)
            cache[level] = tuple(homogeneous_rules(r, L.ny, self._sweep_rule_dtype(L), L.device)
                                 for r in self._rules[level])
        return cache[level]

    def solve_refined(self, f=None, tol=1e-8, inner_tol=None, check_every=200, max_sweeps=10 ** 7, max_outer=30,
                      external_force=None, stall_checks=20):
        """Pseudo-time iteration to an FP64 relative residual ``tol`` with the
        bulk of the sweeps in FP32 (mixed-precision iterative refinement,
        ``refine.py``): FP64 master state and defect sweeps, FP32 correction
        sweeps.  Single-level FP32 solvers ('f32/f32'); an FP64 twin of the
        solver (same class and keywords) computes the defects.  Returns
        ``(F, sweeps, relative_residual)`` with F the FP64 populations;
        ``self.refine_stats`` holds the outer/inner breakdown."""
        from .refine import CorrectionLoop, refine, twin64
        L = self._L(0)
        if L.dtype != torch.float32:
            raise _lib.XlbbError("solve_refined runs its bulk sweeps in FP32: use precision 'f32/f32'")
        if self.levels != 1:
            raise NotImplementedError("solve_refined: single-level solvers (MG_levels=1)")
        if "_twin" not in self.__dict__:
            self._twin = twin64(self)
        twin = self._twin
        T = twin._L(0)
        F = twin.assign_fields_sharded() if f is None else T.field(f, 8).clone()
        ext = T.field(external_force, 2)
        key = ("refine", int(check_every))
        cache = self.__dict__.setdefault("_loops", {})
        if key not in cache:
            cache[key] = CorrectionLoop(self, check_every, 8, lambda a, b, sq, r: self._sweep(
                a, 0, 0.0, 1.0, resid=r, out=b, sumsq=sq, sumsq_diff=True, homogeneous=True))
        loop = cache[key]
        D = T.empty(8)
        sc = torch.zeros(1, dtype=torch.float64, device=L.device)

        def defect(F):
            twin._sweep(F, 0, 1.0, -1.0, fext=ext, out=D, sumsq=True)     # F - S(F)
            twin._reduce_partials(sc)
            return D.clone(), float(sc[0]) ** 0.5
        F, stats = refine(defect, loop, F, tol, inner_tol, max_sweeps, max_outer, stall_checks,
                          lambda x: T.field(x, 8))
        self.refine_stats = stats
        return F, stats["sweeps_f32"] + stats["sweeps_f64"], stats["relative_residual"]

    def _reduce_partials(self, out_scalar):
        _lib.check(_lib.lib().xlbb_reduce_sum(self._partials.data_ptr(), self._n_partials, out_scalar.data_ptr(),
                                              _lib.stream_ptr()), "xlbb_reduce_sum")
        return out_scalar

    # ------------------------------------------------------------------ tolerance drivers
    def solve(self, f=None, tol=1e-8, check_every=100, max_sweeps=10 ** 7, external_force=None, stall_checks=20):
        """Pseudo-time iteration to a relative residual ``||f^{n+1} - f^n|| /
        ||f^1 - f^0|| < tol`` (FP64 norms on the device).  Single level: sweeps
        run as one CUDA graph of ``check_every`` sweeps between host checks.
        Multigrid: V-cycles until the level-0 residual norm drops by ``tol``.
        Returns ``(f, iterations, relative_residual)``."""
        f = self.assign_fields_sharded() if f is None else self._f(f)
        self.stalled = False
        if self.levels > 1:
            f, r0 = self.step(f, 0, external_force=external_force)
            r0 = float(r0)
            require_finite(r0, "level-0 residual norm of the first V-cycle", 1)
            state = {"f": f, "it": 1}

            def vcycle():
                state["f"], r = self.step(state["f"], state["it"], external_force=external_force)
                state["it"] += 1
                return 1, (float(r) / r0 if r0 > 0 else 0.0)
            it, rel, _ = iterate_to_tolerance(vcycle, tol, max_sweeps - 1, what="relative V-cycle residual")
            return state["f"], it + 1, rel
        loop = self._elastic_loop(check_every, external_force)
        r0 = loop.first(f)
        require_finite(r0, "first sweep's residual norm", 1)

        def replay():
            loop.replay()
            return loop.n, ((float(loop.sumsq[0]) ** 0.5) / r0 if r0 > 0 else 0.0)
        it, rel, self.stalled = iterate_to_tolerance(replay, tol, max_sweeps - 1, stall_checks)
        return loop.result, it + 1, rel

    def _elastic_loop(self, n, external_force):
        """The ``ElasticLoop`` of ``n`` sweeps, captured once per solver and
        reused (a new external force is copied into its buffer in place)."""
        cache = self.__dict__.setdefault("_loops", {})
        key = (int(n), external_force is None)
        loop = cache.get(key)
        if loop is None:
            loop = cache[key] = ElasticLoop(self, n, external_force)
        elif external_force is not None:
            loop.ext.copy_(self._L().field(external_force, 2))
        return loop

    def _restrict_full(self, res, level):
        Lf, Lc = self._L(level), self._L(level + 1)
        rc = Lc.empty(8)
        m = self.mg_BCs
        _lib.check(_lib.lib().xlbb_restrict(_lib.dtype_code(Lf.dtype), _lib.dtype_code(Lc.dtype), Lf.grid(), Lc.grid(), 8, int(m["left"]), int(m["right"]),
                                            int(m["bottom"]), int(m["top"]), res.data_ptr(), rc.data_ptr(),
                                            _lib.stream_ptr()), "xlbb_restrict")
        return rc

    def _prolong_add(self, fc, ff, level):
        Lf, Lc = self._L(level), self._L(level + 1)
        m = self.mg_BCs
        _lib.check(_lib.lib().xlbb_prolong_add(_lib.dtype_code(Lf.dtype), _lib.dtype_code(Lc.dtype), Lf.grid(), Lc.grid(), 8, int(m["left"]), int(m["right"]),
                                               int(m["bottom"]), int(m["top"]), fc.data_ptr(), ff.data_ptr(),
                                               _lib.stream_ptr()), "xlbb_prolong_add")

    def _ext_force(self, external_force, nonlinear_force, f, level):
        """external_force + nonlinear_force(f) on level ``level`` (``:1259-1265``)."""
        L = self._L(level)
        if callable(nonlinear_force):
            if hasattr(nonlinear_force, "evaluate"):
                return nonlinear_force.evaluate(self, f, level, external_force)
            nl = L.field(nonlinear_force(f), 2)
            return nl if external_force is None else L.field(external_force + nl, 2)
        return external_force

    def step(self, f_poststreaming, timestep, return_fpost=False, external_force=None, nonlinear_force=None):
        """``:1128-1167``."""
        if self.levels == 1:
            f = self._f(f_poststreaming)
            ext = self._L().field(external_force, 2)
            if callable(nonlinear_force):
                ext = self._ext_force(ext, nonlinear_force, f, 0)
            return self._step(f, timestep, return_fpost, ext)
        return self._mg_step(f_poststreaming, timestep, external_force=external_force,
                             nonlinear_force=nonlinear_force)

    def _step(self, f_poststreaming, timestep, return_fpost=False, external_force=None, level=0):
        """``:1169-1219``: one fused sweep."""
        L = self._L(level)
        f = L.field(f_poststreaming, 8)
        fe = L.field(external_force, 2)
        out = self._sweep(f, level, fext=fe)
        if return_fpost:
            fpost = self.collision(f, fe, level == 0)
            return out, self.apply_bc(fpost, f, timestep, "PostCollision", level)
        return out, None

    def _mg_step(self, f_poststreaming, timestep, level=0, residual=None, external_force=None,
                 nonlinear_force=None):
        """``:1221-1312``: V-cycle.  Smoothing sweeps are ``a=1-gamma, b=gamma``
        fused sweeps, the residual a ``a=1, b=-1`` sweep whose FP64 sum of squares
        over the interior is reduced on the device, restriction / prolongation
        are kernels, the coarse problem starts from zero."""
        L = self._L(level)
        f = L.field(f_poststreaming, 8)
        fe = L.field(external_force, 2)
        g = self.gamma
        for _ in range(self.k_smooth):
            f = self._coupled_sweep(f, level, 1.0 - g, g, residual, fe, nonlinear_force)
        res_norm = None
        if level < self.levels - 1:
            if level == 0:
                ext = self._ext_force(fe, nonlinear_force, f, level)
                res = self._sweep(f, level, 1.0, -1.0, resid=residual, fext=ext, sumsq=True, acc64=self._res64)
            else:
                res = self._coupled_sweep(f, level, 1.0, -1.0, residual, fe, nonlinear_force)
            if level == 0:
                _lib.check(_lib.lib().xlbb_reduce_sum(self._partials.data_ptr(), self._n_partials,
                                                      self._scalar.data_ptr(),
                                                      _lib.stream_ptr()), "xlbb_reduce_sum")
                res_norm = torch.sqrt(self._scalar[0].clone())
            rc = self._restrict_full(res, level)
            fc = self._L(level + 1).zeros(8)
            fc = self._mg_step(fc, timestep, level + 1, rc, nonlinear_force=nonlinear_force)
            self._prolong_add(fc, f, level)
        for _ in range(self.k_smooth):
            f = self._coupled_sweep(f, level, 1.0 - g, g, residual, fe, nonlinear_force)
        if level == 0:
            return f, res_norm
        return f

    def _coupled_sweep(self, f, level, a, b, resid, fe, nonlinear_force):
        """A sweep ``a f + b STEP(f - resid)`` whose external force is ``fe`` plus
        the nonlinear force of its own input.  The poroelastic coupling force
        (``DivGradForce``) is fused into the sweep (``xlbb_elast_sweep_divgrad``:
        one launch, the same values bit for bit) when the sweep qualifies;
        otherwise the force is evaluated first."""
        L = self._L(level)
        if self._fused_coupling and getattr(nonlinear_force, "fusable", False) and not self._sweep_acc64(L):
            out = self._sweep(f, level, a, b, resid=resid, fext=fe, coupling=nonlinear_force)
            if out is not None:
                return out
        ext = self._ext_force(fe, nonlinear_force, f, level)
        return self._sweep(f, level, a, b, resid=resid, fext=ext)

    # ------------------------------------------------------------------ driver
    def run(self, t_max):
        """``:1346-1425``: t_max + 1 steps with I/O through ``output_data``."""
        f = self.assign_fields_sharded()
        start = time.time()
        for timestep in range(0, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            print_iter_flag = self.printInfoRate > 0 and timestep % self.printInfoRate == 0
            if io_flag:
                eta_prev, sigma_prev = self.update_macroscopic(f)
                eta_prev, sigma_prev = gathered(eta_prev), gathered(sigma_prev)
            f, fstar = self.step(f, timestep, return_fpost=self.returnFpost)
            if print_iter_flag:
                print(f"Timestep {timestep} of {t_max} completed")
            if io_flag:
                eta, sigma = self.update_macroscopic(f)
                if isinstance(fstar, torch.Tensor) and fstar.dim() == 0:
                    fstar = float(fstar)
                self.handle_io_timestep(timestep, f, fstar, gathered(eta), gathered(sigma), eta_prev, sigma_prev)
            if self.computeMLUPS and timestep == 1:
                torch.cuda.synchronize()
                start = time.time()
        if self.computeMLUPS:
            torch.cuda.synchronize()
            end = time.time()
            print(f"Domain: {self.nx} x {self.ny}")
            print(f"Number of voxels: {self.nx * self.ny}")
            print(f"MLUPS: {self.nx * self.ny * t_max / (end - start) / 1e6}")
        return f

    def handle_io_timestep(self, timestep, f, fstar, eta, sigma, eta_prev, sigma_prev):
        self.output_data(timestep=timestep, eta=eta, eta_prev=eta_prev, sigma=sigma, sigma_prev=sigma_prev,
                         f_poststreaming=f, f_postcollision=fstar)


class ElasticityBounceBackFullway(BoundaryCondition):
    """``src/elasticity.py:1503-1550``: post-collision full-way bounce-back with an
    optional wall displacement ``eta``."""

    def __init__(self, indices, gridInfo, precision_policy, eta=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ElasticityBounceBackFullway"
        self.implementationStep = "PostCollision"
        self.eta = None if eta is None else np.asarray(eta, dtype=np.float64)

    def apply(self, fout, fin):
        out = _take(fin, self.indices)[..., self.lattice.opp_indices]
        if self.eta is None:
            return out
        c = np.array(self.lattice.c, dtype=np.float64)
        return out + 6.0 * self.lattice.w.astype(np.float64) * np.dot(self.eta, c)


class ElasticityBounceBack(BoundaryCondition):
    """``src/elasticity.py:1552-1646``: halfway bounce-back (Dirichlet)."""

    def __init__(self, indices, gridInfo, precision_policy, eta=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ElasticityBounceBack"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.eta = None if eta is None else np.asarray(eta, dtype=np.float64)

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        first = self._halfway_index_shift(boundaryMask)
        nbd = len(self.indices[0])
        if nbd_orig != nbd and self.eta is not None:
            if self.eta.shape == (self.lattice.d,):
                self.eta = np.tile(self.eta, (nbd, 1))
            else:
                print("WARNING: Assuming a correct displacement vector to impose at the BC cells!")
                self.eta = self.eta[first]
        elif self.eta is not None and self.eta.shape == (self.lattice.d,):
            self.eta = np.tile(self.eta, (nbd, 1))

    def impose_boundary_displacement(self, fbd, bindex):
        c = np.array(self.lattice.c, dtype=np.float64)
        cu = 6.0 * self.lattice.w.astype(np.float64) * np.dot(self.eta, c)
        return _at_add(fbd, (bindex, self.imissing), cu[bindex, self.imissing])

    def apply(self, fout, fin):
        nbd = len(self.indices[0])
        bindex = np.arange(nbd)[:, None]
        fbd = np.array(_take(fout, self.indices))
        _at_set(fbd, (bindex, self.imissing), _take(fin, self.indices)[bindex, self.iknown])
        if self.eta is not None:
            fbd = self.impose_boundary_displacement(fbd, bindex)
        return fbd


class ElasticityAntiBounceBack(BoundaryCondition):
    """``src/elasticity.py:1648-1750``: halfway anti-bounce-back (Neumann /
    traction ``T``)."""

    def __init__(self, indices, gridInfo, precision_policy, T=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ElasticityAntiBounceBack"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.T = None if T is None else np.asarray(T, dtype=np.float64)

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        first = self._halfway_index_shift(boundaryMask)
        nbd = len(self.indices[0])
        if nbd_orig != nbd and self.T is not None:
            if self.T.shape == (self.lattice.d,):
                self.T = np.tile(self.T, (nbd, 1))
            else:
                print("WARNING: Assuming a correct normal stress vector to impose at the BC cells!")
                self.T = self.T[first]
        elif self.T is not None and self.T.shape == (self.lattice.d,):
            self.T = np.tile(self.T, (nbd, 1))

    def get_missing_mask(self, boundaryMask):
        if self.T is not None:
            normals = self.get_normals(boundaryMask)
            T = self.T
            if np.all(normals[:, 0] == -1):
                self.i_update = (0, 4, 7)
                self.T_update = np.stack((T[:, 0], 0.5 * T[:, 1], -0.5 * T[:, 1]), axis=-1)
            elif np.all(normals[:, 0] == 1):
                self.i_update = (2, 5, 6)
                self.T_update = np.stack((-T[:, 0], 0.5 * T[:, 1], -0.5 * T[:, 1]), axis=-1)
            elif np.all(normals[:, 1] == -1):
                self.i_update = (1, 4, 5)
                self.T_update = np.stack((T[:, 1], 0.5 * T[:, 0], -0.5 * T[:, 0]), axis=-1)
            elif np.all(normals[:, 1] == 1):
                self.i_update = (3, 6, 7)
                self.T_update = np.stack((-T[:, 1], -0.5 * T[:, 0], 0.5 * T[:, 0]), axis=-1)
            else:
                raise NotImplementedError
        return super().get_missing_mask(boundaryMask)

    def apply(self, fout, fin):
        fbd = np.array(_take(fout, self.indices))
        fbd[self.imissingMask] = -_take(fin, self.indices)[self.iknownMask]
        if self.T is not None:
            fbd[:, list(self.i_update)] += self.T_update
        return fbd


class ElasticLoop:
    """``n`` plain elasticity sweeps captured once as a CUDA graph; the last sweep
    reduces the FP64 residual sum((f_n - f_{n-1})^2) into ``sumsq``."""

    def __init__(self, solver, n, external_force=None):
        L = solver._L(0)
        self.solver, self.n = solver, int(n) + (int(n) % 2)   # even: the result lands in ``state``
        self.state, self._other = L.empty(8), L.empty(8)
        self.ext = None                       # owned buffer: the graph reads it by address
        if external_force is not None:
            self.ext = L.empty(2)
            self.ext.copy_(L.field(external_force, 2))
        self.sumsq = torch.zeros(1, dtype=torch.float64, device=L.device)
        self.launches_per_replay = self.n + 1
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._body()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()
        self.result = self.state if self.n % 2 == 0 else self._other

    def _body(self):
        a, b = self.state, self._other
        for k in range(self.n):
            self.solver._sweep(a, 0, fext=self.ext, out=b, sumsq=(k == self.n - 1), sumsq_diff=True)
            a, b = b, a
        self.solver._reduce_partials(self.sumsq)

    def first(self, f0):
        """One sweep from ``f0`` into ``state``; returns ||f^1 - f^0|| (FP64)."""
        self.solver._sweep(f0, 0, fext=self.ext, out=self.state, sumsq=True, sumsq_diff=True)
        self.solver._reduce_partials(self.sumsq)
        return float(self.sumsq[0]) ** 0.5

    def replay(self):
        self.graph.replay()
        return self.result
