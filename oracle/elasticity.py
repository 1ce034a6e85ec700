"""D2Q8 linear-elasticity LBM with geometric multigrid (oracle).

Restates ``src/elasticity.py`` (``LBMElasticity`` and its three boundary
conditions) in NumPy.  Only what the Biot hot path uses is kept: 2D, one device,
no I/O side effects beyond the ``output_data`` hook.
"""
import numpy as np

from . import jaxsem
from .boundary_conditions import (BoundaryCondition, create_grid_mask, solid_voxels,
                                  stream, apply_bc_list)
from .lattice import Policy


def coarsen_field(a, mg_bcs):
    """Extension without a reference counterpart (the reference's Lame
    parameters are uniform): the material field of the next coarser level.
    Interior: mean of each 2 x 2 fine block (the block the restriction sums);
    rows / columns kept by ``MG_BCs``: mean of the fine pair along them;
    corners: copied."""
    l, r, b, t = (int(mg_bcs[k]) for k in ("left", "right", "bottom", "top"))
    nx, ny = a.shape
    nxc, nyc = (nx - l - r) // 2 + l + r, (ny - b - t) // 2 + b + t
    out = np.empty((nxc, nyc), dtype=a.dtype)
    for X in range(nxc):
        for Y in range(nyc):
            xin, yin = l <= X < nxc - r, b <= Y < nyc - t
            xs = [l + 2 * (X - l), l + 2 * (X - l) + 1] if xin else [0 if X < l else nx - 1]
            ys = [b + 2 * (Y - b), b + 2 * (Y - b) + 1] if yin else [0 if Y < b else ny - 1]
            out[X, Y] = np.mean([a[x, y] for x in xs for y in ys])
    return out


class LBMElasticity:
    """``src/elasticity.py:30-1501``.

    Extension: ``lambda_field`` / ``mu_field`` (shape (nx, ny)) give per-cell
    Lame parameters; coarse levels use ``coarsen_field``.  With uniform fields
    every formula reduces to the reference's."""

    def __init__(self, **kwargs):
        self.lamda = kwargs.get("lambda")
        self.mu = kwargs.get("mu")
        self.nx, self.ny, self.nz = kwargs.get("nx"), kwargs.get("ny"), kwargs.get("nz")
        mg = {"left": False, "right": False, "bottom": False, "top": False, "front": False, "back": False}
        mg.update(kwargs.get("MG_BCs", {}))
        self.mg_BCs = mg
        self.levels = kwargs.get("MG_levels", 1)
        den = 2 ** (self.levels - 1)
        if ((self.nx - int(mg["left"]) - int(mg["right"])) % den
                or (self.ny - int(mg["bottom"]) - int(mg["top"])) % den):
            raise ValueError("nx,ny,nz (-BCs) must be divisible by 2**(levels-1)")
        self.gamma = kwargs.get("MG_relaxation", 0.75)
        self.k_smooth = kwargs.get("MG_n_smoothing", 2)
        self.precision = kwargs.get("precision")
        self.precisionPolicy = Policy(self.precision)
        self.lattice = kwargs.get("lattice")
        self.ioRate = kwargs.get("io_rate", 0)
        self.printInfoRate = kwargs.get("print_info_rate", 100)
        self.returnFpost = kwargs.get("return_fpost", False)
        self.c, self.q, self.w, self.dim = self.lattice.c, self.lattice.q, self.lattice.w, self.lattice.d
        self._create_transfer_matrices()
        self.gridInfo = {"nx": self.nx, "ny": self.ny, "nz": self.nz, "dim": 2, "lattice": self.lattice}
        self.boundingBoxIndices = self.bounding_box_indices()
        self._create_boundary_data()
        self.force = self.get_force()
        if self.force is not None:
            self.force = np.asarray(self.force, dtype=self.precisionPolicy.compute_dtype)
        self._fields = None
        lf, mf = kwargs.get("lambda_field"), kwargs.get("mu_field")
        if lf is not None:
            lam = np.asarray(lf, dtype=np.float64).reshape(self.nx, self.ny)
            mu = np.asarray(mf, dtype=np.float64).reshape(self.nx, self.ny)
            self._fields = [(lam, mu)]
            for _ in range(1, self.levels):
                lam, mu = coarsen_field(lam, self.mg_BCs), coarsen_field(mu, self.mg_BCs)
                self._fields.append((lam, mu))

    def _material(self, shape):
        """(lambda, mu) for an array of ``shape``: scalars, or (nx, ny, 1) fields
        of the level whose grid has that shape."""
        if self._fields is None:
            return self.lamda, self.mu
        for level in range(self.levels):
            if tuple(shape[:2]) == self.grid_size(level):
                lam, mu = self._fields[level]
                dt = self.precisionPolicy.compute_dtype
                return lam[..., None].astype(dt), mu[..., None].astype(dt)
        raise ValueError("no level has this shape")

    def _m_to_f_apply(self, m, lam, mu):
        """m (..., 7) @ m_to_f with a per-cell ms row when the fields vary."""
        if self._fields is None:
            return np.matmul(m, self.m_to_f)
        g = 1.0 / (12.0 * (lam + mu) - 4.0)
        g = np.where(np.abs(g) > 100, 0.0, g)
        base = self.m_to_f.copy()
        base[2, :] = 0
        hn = np.concatenate([np.broadcast_to(0.25 + 0.5 * g, g.shape[:2] + (4,)),
                             np.broadcast_to(-0.25 * g, g.shape[:2] + (4,))], axis=-1)
        return np.matmul(m, base) + m[..., 2:3] * hn

    # -- setup -------------------------------------------------------------
    def _create_boundary_data(self):
        """``:396-436``."""
        self.BCs = []
        self.BCs_MG = {level: [] for level in range(1, self.levels)}
        self.set_boundary_conditions()
        nx, ny = self.grid_size(0)
        grid_mask = create_grid_mask(nx, ny, self.lattice, solid_voxels(self.BCs))
        for bc in self.BCs:
            bc.create_local_mask_and_normal_arrays(grid_mask)
        for level in range(1, self.levels):
            nx, ny = self.grid_size(level)
            grid_mask = create_grid_mask(nx, ny, self.lattice, solid_voxels(self.BCs_MG[level]))
            for bc in self.BCs_MG[level]:
                bc.create_local_mask_and_normal_arrays(grid_mask)

    def grid_size(self, level=0):
        """``:501-529``."""
        if level == 0:
            return self.nx, self.ny
        nxb = int(self.mg_BCs["left"]) + int(self.mg_BCs["right"])
        nyb = int(self.mg_BCs["bottom"]) + int(self.mg_BCs["top"])
        return (self.nx - nxb) // 2 ** level + nxb, (self.ny - nyb) // 2 ** level + nyb

    def grid_info(self, level=0):
        nx, ny = self.grid_size(level)
        return {"nx": nx, "ny": ny, "nz": self.nz, "dim": 2, "lattice": self.lattice}

    def bounding_box_indices(self, level=0):
        """``:563-589``."""
        nx, ny = self.grid_size(level)
        return {"bottom": np.array([[i, 0] for i in range(nx)], dtype=int),
                "top": np.array([[i, ny - 1] for i in range(nx)], dtype=int),
                "left": np.array([[0, i] for i in range(ny)], dtype=int),
                "right": np.array([[nx - 1, i] for i in range(ny)], dtype=int)}

    def distributed_array_init(self, shape, type, init_val=0, sharding=None):
        return np.broadcast_to(np.asarray(init_val, dtype=type), shape).astype(type)

    def _create_transfer_matrices(self):
        """``:805-848``."""
        g = 1.0 / (12.0 * (self.lamda + self.mu) - 4.0)
        if abs(g) > 100:
            g = 0.0
        dt = self.precisionPolicy.compute_dtype
        self.f_to_m = np.array([[1, 0, -1, 0, 1, -1, -1, 1],
                                [0, 1, 0, -1, 1, 1, -1, -1],
                                [1, 1, 1, 1, 2, 2, 2, 2],
                                [1, -1, 1, -1, 0, 0, 0, 0],
                                [0, 0, 0, 0, 1, -1, 1, -1]], dtype=dt).T
        h = 0.25 + 0.5 * g
        n = -0.25 * g
        self.m_to_f = np.array([[0.5, 0, h, 0.25, 0, -0.5, 0],
                                [0, 0.5, h, -0.25, 0, 0, -0.5],
                                [-0.5, 0, h, 0.25, 0, 0.5, 0],
                                [0, -0.5, h, -0.25, 0, 0, 0.5],
                                [0, 0, n, 0, 0.25, 0.25, 0.25],
                                [0, 0, n, 0, -0.25, -0.25, 0.25],
                                [0, 0, n, 0, 0.25, -0.25, -0.25],
                                [0, 0, n, 0, -0.25, 0.25, -0.25]], dtype=dt).T

    # -- hooks ---------------------------------------------------------------
    def set_boundary_conditions(self):
        pass

    def get_force(self):
        return None

    def initialize_macroscopic_fields(self):
        return None, None

    def output_data(self, **kwargs):
        pass

    # -- physics -----------------------------------------------------------
    def assign_fields_sharded(self):
        """``:647-679``."""
        eta0, sigma0 = self.initialize_macroscopic_fields()
        if eta0 is None or sigma0 is None:
            return np.zeros((self.nx, self.ny, self.q), dtype=self.precisionPolicy.output_dtype)
        return self.equilibrium(eta0, sigma0)

    def equilibrium(self, eta, sigma, cast_output=True, external_force=None):
        """``:909-957``."""
        if cast_output:
            eta, sigma = self.precisionPolicy.cast_to_compute((eta, sigma))
        if self.force is not None:
            eta = eta - 0.5 * self.force
        if external_force is not None:
            eta = eta - 0.5 * external_force
        lam, mu = self._material(np.shape(sigma))
        cs = -1.0 - 1 / (3 * (lam + mu))
        ms = (sigma[..., 0:1] + sigma[..., 2:3]) * cs
        cd = -1.0 - 1 / (6 * mu)
        md = (sigma[..., 0:1] - sigma[..., 2:3]) * cd
        m11 = sigma[..., 1:2] * cd
        m = np.concatenate((eta, ms, md, m11, eta / 3.0), axis=-1)
        feq = self._m_to_f_apply(m, lam, mu)
        return self.precisionPolicy.cast_to_output(feq) if cast_output else feq

    def collision(self, f, external_force, use_force=True):
        """``:959-1000`` (the four force branches)."""
        f = self.precisionPolicy.cast_to_compute(f)
        external_force = self.precisionPolicy.cast_to_compute(external_force)
        m = np.matmul(f, self.f_to_m)
        lam, mu = self._material(f.shape)
        cs = (3 * (lam + mu) - 1) / (3 * (lam + mu) + 1)
        cd = (6 * mu - 1) / (6 * mu + 1)
        if use_force and self.force is not None and external_force is not None:
            force = self.force + external_force
        elif external_force is not None:
            force = external_force
        elif use_force and self.force is not None:
            force = self.force
        else:
            force = None
        if force is not None:
            m = np.concatenate([m[..., 0:2] + force, m[..., 2:3] * cs, m[..., 3:5] * cd,
                                m[..., 0:2] / 3.0 + force / 6.0], axis=-1)
        else:
            m = np.concatenate([m[..., 0:2], m[..., 2:3] * cs, m[..., 3:5] * cd,
                                m[..., 0:2] / 3.0], axis=-1)
        return self.precisionPolicy.cast_to_output(self._m_to_f_apply(m, lam, mu))

    def update_macroscopic(self, f, external_force=None):
        """``:1002-1038``."""
        m = np.matmul(f, self.f_to_m)
        eta = m[..., 0:2]
        if self.force is not None:
            eta = eta + 0.5 * self.force
        if external_force is not None:
            eta = eta + 0.5 * external_force
        lam, mu = self._material(f.shape)
        if self._fields is not None:
            lam, mu = lam[..., 0], mu[..., 0]
        cs = -1.5 * (lam + mu) / (3 * (lam + mu) + 1)
        ms = m[..., 2] * cs
        cd = -3 * mu / (6 * mu + 1)
        md = m[..., 3] * cd
        sigma = np.stack((ms + md, (2 * cd) * m[..., 4], ms - md), axis=-1)
        return eta, sigma

    def update_divergence(self, f):
        """``:1040-1058``."""
        lam, mu = self._material(f.shape)
        return (-1.5 / (3 * (lam + mu) + 1)) * np.matmul(f, self.f_to_m[:, 2:3])

    def streaming(self, f):
        return stream(f, self.c)

    def _bcs(self, level):
        return self.BCs if level == 0 else self.BCs_MG[level]

    def _step(self, f_poststreaming, timestep, return_fpost=False, external_force=None, level=0):
        """``:1169-1219``."""
        f_postcollision = self.collision(f_poststreaming, external_force, level == 0)
        f_postcollision = apply_bc_list(self._bcs(level), f_postcollision, f_poststreaming, "PostCollision")
        f_new = self.streaming(f_postcollision)
        f_new = apply_bc_list(self._bcs(level), f_new, f_postcollision, "PostStreaming")
        return (f_new, f_postcollision) if return_fpost else (f_new, None)

    def step(self, f_poststreaming, timestep, return_fpost=False, external_force=None, nonlinear_force=None):
        """``:1128-1167``."""
        if self.levels == 1:
            if callable(nonlinear_force):
                external_force = external_force + nonlinear_force(f_poststreaming)
            return self._step(f_poststreaming, timestep, return_fpost, external_force)
        return self._mg_step(f_poststreaming, timestep, external_force=external_force,
                             nonlinear_force=nonlinear_force)

    def _interior(self, shape):
        return (slice(int(self.mg_BCs["left"]), shape[0] - int(self.mg_BCs["right"])),
                slice(int(self.mg_BCs["bottom"]), shape[1] - int(self.mg_BCs["top"])))

    def substract_residual(self, f, residual):
        """``:1314-1344``."""
        if residual is None:
            return f
        f = np.array(f, copy=True)
        f[self._interior(f.shape)] += -residual
        return f

    def _ext(self, external_force, nonlinear_force, f):
        if callable(nonlinear_force):
            if external_force is not None:
                return external_force + nonlinear_force(f)
            return nonlinear_force(f)
        return external_force

    def _mg_step(self, f, timestep, level=0, residual=None, external_force=None, nonlinear_force=None):
        """``:1221-1312``: damped pre/post smoothing, residual, restriction,
        coarse recursion from zero, prolongation; level 0 returns the L2 norm
        of the interior residual."""
        g = self.gamma
        for _ in range(self.k_smooth):
            ext = self._ext(external_force, nonlinear_force, f)
            f = (1 - g) * f + g * self._step(self.substract_residual(f, residual), timestep, False, ext, level)[0]
        res = None
        if level < self.levels - 1:
            ext = self._ext(external_force, nonlinear_force, f)
            res = f - self._step(self.substract_residual(f.copy(), residual), timestep, False, ext, level)[0]
            res_coarse = self._restrict(res)
            f_coarse = np.zeros((*self.grid_size(level + 1), self.q), dtype=self.precisionPolicy.compute_dtype)
            f_coarse = self._mg_step(f_coarse, timestep, level + 1, res_coarse, nonlinear_force=nonlinear_force)
            f = np.array(f, copy=True)
            f[self._interior(f.shape)] += self._prolong(f_coarse)
        for _ in range(self.k_smooth):
            ext = self._ext(external_force, nonlinear_force, f)
            f = (1 - g) * f + g * self._step(self.substract_residual(f, residual), timestep, False, ext, level)[0]
        if level == 0:
            return f, np.linalg.norm(res[self._interior(res.shape)].ravel())
        return f

    def _restrict(self, f):
        """``:850-865``: 2x2 block SUM over the interior."""
        s = f[self._interior(f.shape)]
        return s[0::2, 0::2] + s[0::2, 1::2] + s[1::2, 0::2] + s[1::2, 1::2]

    def _prolong(self, f):
        """``:878-894``: piecewise-constant injection of the coarse interior."""
        s = f[self._interior(f.shape)]
        return np.repeat(np.repeat(s, 2, axis=0), 2, axis=1)

    def run(self, t_max):
        """``:1346-1425`` (t_max + 1 sweeps; I/O through ``output_data``)."""
        f = self.assign_fields_sharded()
        for timestep in range(0, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            if io_flag:
                eta_prev, sigma_prev = self.update_macroscopic(f)
            f, fstar = self.step(f, timestep, return_fpost=self.returnFpost)
            if io_flag:
                eta, sigma = self.update_macroscopic(f)
                self.output_data(timestep=timestep, eta=eta[None], eta_prev=eta_prev[None],
                                 sigma=sigma[None], sigma_prev=sigma_prev[None],
                                 f_poststreaming=f, f_postcollision=fstar)
        return f


class ElasticityBounceBackFullway(BoundaryCondition):
    """``src/elasticity.py:1503-1550`` (post-collision, non-solid)."""

    def __init__(self, indices, gridInfo, precision_policy, eta=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ElasticityBounceBackFullway"
        self.implementationStep = "PostCollision"
        self.eta = eta

    def apply(self, fout, fin):
        out = jaxsem.gather(fin, self.indices)[..., self.lattice.opp_indices]
        if self.eta is None:
            return out
        c = np.array(self.lattice.c, dtype=self.precisionPolicy.compute_dtype)
        return out + 6.0 * self.lattice.w * np.dot(self.eta, c)


class ElasticityBounceBack(BoundaryCondition):
    """``src/elasticity.py:1552-1646`` (halfway Dirichlet, post-streaming)."""

    def __init__(self, indices, gridInfo, precision_policy, eta=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ElasticityBounceBack"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.eta = None if eta is None else np.asarray(eta)

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        _, first = self.halfway_shift(boundaryMask)
        nbd = len(self.indices[0])
        if nbd_orig != nbd and self.eta is not None:
            if self.eta.shape == (self.lattice.d,):
                self.eta = np.tile(self.eta, (nbd, 1))
            else:
                self.eta = self.eta[first]
        elif self.eta is not None and self.eta.shape == (self.lattice.d,):
            self.eta = np.tile(self.eta, (nbd, 1))

    def apply(self, fout, fin):
        nbd = len(self.indices[0])
        bindex = np.arange(nbd)[:, None]
        fbd = jaxsem.gather(fout, self.indices)
        fbd = jaxsem.scatter_set(fbd, (bindex, self.imissing),
                                 jaxsem.gather(fin, self.indices)[bindex, self.iknown])
        if self.eta is not None:
            c = np.array(self.lattice.c, dtype=self.precisionPolicy.compute_dtype)
            cu = 6.0 * self.lattice.w * np.dot(self.eta, c)
            fbd = jaxsem.scatter_add(fbd, (bindex, self.imissing), cu[bindex, self.imissing])
        return fbd


class ElasticityAntiBounceBack(BoundaryCondition):
    """``src/elasticity.py:1648-1750`` (halfway Neumann / traction)."""

    def __init__(self, indices, gridInfo, precision_policy, T=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ElasticityAntiBounceBack"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.T = None if T is None else np.asarray(T)

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        _, first = self.halfway_shift(boundaryMask)
        nbd = len(self.indices[0])
        if nbd_orig != nbd and self.T is not None:
            if self.T.shape == (self.lattice.d,):
                self.T = np.tile(self.T, (nbd, 1))
            else:
                self.T = self.T[first]
        elif self.T is not None and self.T.shape == (self.lattice.d,):
            self.T = np.tile(self.T, (nbd, 1))

    def get_missing_mask(self, boundaryMask):
        if self.T is not None:
            nrm = self.get_normals(boundaryMask)
            T = self.T
            if np.all(nrm[:, 0] == -1):
                self.i_update = (0, 4, 7)
                self.T_update = np.stack((T[:, 0], 0.5 * T[:, 1], -0.5 * T[:, 1]), axis=-1)
            elif np.all(nrm[:, 0] == 1):
                self.i_update = (2, 5, 6)
                self.T_update = np.stack((-T[:, 0], 0.5 * T[:, 1], -0.5 * T[:, 1]), axis=-1)
            elif np.all(nrm[:, 1] == -1):
                self.i_update = (1, 4, 5)
                self.T_update = np.stack((T[:, 1], 0.5 * T[:, 0], -0.5 * T[:, 0]), axis=-1)
            elif np.all(nrm[:, 1] == 1):
                self.i_update = (3, 6, 7)
                self.T_update = np.stack((-T[:, 1], -0.5 * T[:, 0], 0.5 * T[:, 0]), axis=-1)
            else:
                raise NotImplementedError
        return super().get_missing_mask(boundaryMask)

    def apply(self, fout, fin):
        fbd = jaxsem.gather(fout, self.indices)
        fbd = jaxsem.bool_mask_set(fbd, self.imissingMask,
                                   -jaxsem.gather(fin, self.indices)[self.iknownMask])
        if self.T is not None:
            fbd = _add_cols(fbd, self.i_update, self.T_update)
        return fbd


def _add_cols(fbd, cols, vals):
    """``fbd.at[:, cols].add(vals)`` with distinct columns."""
    out = np.array(fbd, copy=True)
    out[:, list(cols)] += vals
    return out
