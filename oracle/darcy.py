"""D2Q9 advection-diffusion-reaction BGK (Darcy pressure) LBM (oracle).

Restates ``src/darcy.py`` and the ``LBMBase`` pieces it uses
(``src/base.py:44-146,351-372,528-559,686-724,776-806``).

Extension beyond the reference (documented, used only where the reference
cannot speak): ``omega`` may be a per-cell array of shape (nx, ny, 1).  For a
scalar ``omega`` every expression is the reference's.
"""
import numpy as np

from . import jaxsem
from .boundary_conditions import (BoundaryCondition, BounceBackHalfway, create_grid_mask,
                                  solid_voxels, stream, apply_bc_list)
from .lattice import Policy


class AdvectionDiffusionReactionBGK:
    """``src/darcy.py:22-296`` on top of ``src/base.py:30-146``."""

    def __init__(self, **kwargs):
        self.omega = kwargs.get("omega")
        self.nx, self.ny, self.nz = kwargs.get("nx"), kwargs.get("ny"), kwargs.get("nz")
        self.precision = kwargs.get("precision")
        self.precisionPolicy = Policy(self.precision)
        self.lattice = kwargs.get("lattice")
        self.ioRate = kwargs.get("io_rate", 0)
        self.returnFpost = kwargs.get("return_fpost", False)
        self.c, self.q, self.w, self.dim = self.lattice.c, self.lattice.q, self.lattice.w, self.lattice.d
        self.sharding = None
        self.gridInfo = {"nx": self.nx, "ny": self.ny, "nz": self.nz, "dim": 2, "lattice": self.lattice}
        self.boundingBoxIndices = self.bounding_box_indices()
        self._create_boundary_data()
        self.force = None
        self.vel = kwargs.get("vel", None)
        self.source = self.get_source()
        if self.source is not None:
            self.source = np.asarray(self.source, dtype=self.precisionPolicy.compute_dtype)

    def bounding_box_indices(self):
        """``src/base.py:451-470``."""
        nx, ny = self.nx, self.ny
        return {"bottom": np.array([[i, 0] for i in range(nx)], dtype=int),
                "top": np.array([[i, ny - 1] for i in range(nx)], dtype=int),
                "left": np.array([[0, i] for i in range(ny)], dtype=int),
                "right": np.array([[nx - 1, i] for i in range(ny)], dtype=int)}

    def _create_boundary_data(self):
        """``src/base.py:351-372``."""
        self.BCs = []
        self.set_boundary_conditions()
        grid_mask = create_grid_mask(self.nx, self.ny, self.lattice, solid_voxels(self.BCs))
        for bc in self.BCs:
            bc.create_local_mask_and_normal_arrays(grid_mask)

    def distributed_array_init(self, shape, type, init_val=0, sharding=None):
        return np.broadcast_to(np.asarray(init_val, dtype=type), shape).astype(type)

    # hooks
    def set_boundary_conditions(self):
        pass

    def get_source(self):
        return None

    def initialize_macroscopic_fields(self):
        return None, None

    def output_data(self, **kwargs):
        pass

    def assign_fields_sharded(self):
        """``src/base.py:528-559``: default populations are the weights."""
        rho0, u0 = self.initialize_macroscopic_fields()
        shape = (self.nx, self.ny, self.q)
        if rho0 is None or u0 is None:
            return np.broadcast_to(self.w.astype(self.precisionPolicy.output_dtype), shape).copy()
        return self.equilibrium(rho0, u0)

    def equilibrium(self, rho, u, cast_output=True):
        """``src/base.py:686-724``."""
        if cast_output:
            rho, u = self.precisionPolicy.cast_to_compute((rho, u))
        c = np.array(self.c, dtype=self.precisionPolicy.compute_dtype)
        cu = 3.0 * np.dot(u, c)
        usqr = 1.5 * np.sum(np.square(u), axis=-1, keepdims=True)
        feq = rho * self.w * (1.0 + cu * (1.0 + 0.5 * cu) - usqr)
        return self.precisionPolicy.cast_to_output(feq) if cast_output else feq

    def streaming(self, f):
        return stream(f, self.c)

    def update_macroscopic(self, f, external_source=None, gradient=False):
        """``src/darcy.py:36-73``."""
        if self.source is not None and external_source is not None:
            rho = np.sum(f, axis=-1, keepdims=True) + 0.5 * (self.source + external_source)
        elif self.source is not None:
            rho = np.sum(f, axis=-1, keepdims=True) + 0.5 * self.source
        elif external_source is not None:
            rho = np.sum(f, axis=-1, keepdims=True) + 0.5 * external_source
        else:
            rho = np.sum(f, axis=-1, keepdims=True)
        if gradient:
            c = np.array(self.c, dtype=self.precisionPolicy.compute_dtype).T
            if np.ndim(self.omega) == 0:
                grad = np.dot(f, (-3 * self.omega) * c)
            else:
                grad = (-3 * self.omega) * np.dot(f, c)
            return rho, grad
        return rho

    def gradient(self, q, scale=1.0):
        """``src/darcy.py:75-104``: isotropic 9-point gradient of a scalar field
        with the (anti-)bounce-back ADR conditions applied to the shifted copies.
        On arrays smaller than the fine grid the fine BC indices are clamped on
        gather and dropped on scatter, as JAX does."""
        p_in = np.tile(q, self.q)
        p_out = self.streaming(p_in)
        for bc in self.BCs:
            if bc.name in ("ADR_Neumann_BounceBack", "ADR_AntiBounceBack"):
                p_out = jaxsem.scatter_set(p_out, bc.indices, bc.apply(p_out, p_in))
        return np.matmul(p_out, -3 * scale * self.w[..., None] * self.c.T)

    def collision(self, f, external_source=None):
        """``src/darcy.py:106-129``."""
        f = self.precisionPolicy.cast_to_compute(f)
        rho = self.update_macroscopic(f, external_source)
        feq = rho * self.w
        fneq = f - feq
        fout = f - self.omega * fneq
        if self.source is not None and external_source is not None:
            fout = fout + (self.source + external_source) * ((1 - 0.5 * self.omega) * self.w)
        elif self.source is not None:
            fout = fout + self.source * ((1 - 0.5 * self.omega) * self.w)
        elif external_source is not None:
            fout = fout + external_source * ((1 - 0.5 * self.omega) * self.w)
        return self.precisionPolicy.cast_to_output(fout)

    def step(self, f_poststreaming, timestep, return_fpost=False, external_source=None):
        """``src/darcy.py:131-171``."""
        f_postcollision = self.collision(f_poststreaming, external_source)
        f_postcollision = apply_bc_list(self.BCs, f_postcollision, f_poststreaming, "PostCollision")
        f_new = self.streaming(f_postcollision)
        f_new = apply_bc_list(self.BCs, f_new, f_postcollision, "PostStreaming")
        return (f_new, f_postcollision) if return_fpost else (f_new, None)

    def run(self, t_max):
        """``src/darcy.py:173-252``: t_max steps, output at step 0 and io steps."""
        f = self.assign_fields_sharded()
        if self.ioRate > 0:
            self.output_data(timestep=0, rho=self.update_macroscopic(f)[None], rho_prev=None,
                             f_poststreaming=f, f_postcollision=None)
        for timestep in range(1, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            if io_flag:
                rho_prev = self.update_macroscopic(f)
            f, fstar = self.step(f, timestep, return_fpost=self.returnFpost)
            if io_flag:
                self.output_data(timestep=timestep, rho=self.update_macroscopic(f)[None],
                                 rho_prev=rho_prev[None], f_poststreaming=f, f_postcollision=fstar)
        return f


class ADR_AntiBounceBack(BoundaryCondition):
    """``src/darcy.py:298-392`` (halfway anti-bounce-back, Dirichlet)."""

    def __init__(self, indices, gridInfo, precision_policy, rho=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ADR_AntiBounceBack"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.rho = rho

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        _, first = self.halfway_shift(boundaryMask)
        nbd = len(self.indices[0])
        if nbd_orig != nbd and self.rho is not None:
            if isinstance(self.rho, float) or np.asarray(self.rho).size == 1:
                self.rho = np.full((nbd, 1), self.rho)
            else:
                self.rho = np.asarray(self.rho)[first]

    def apply(self, fout, fin):
        nbd = len(self.indices[0])
        bindex = np.arange(nbd)[:, None]
        fbd = jaxsem.gather(fout, self.indices)
        fbd = jaxsem.scatter_set(fbd, (bindex, self.imissing),
                                 -jaxsem.gather(fin, self.indices)[bindex, self.iknown])
        if self.rho is not None:
            tmp = 2 * self.lattice.w * np.asarray(self.rho)
            tmp = np.broadcast_to(tmp, (nbd, self.lattice.q))
            fbd = jaxsem.scatter_add(fbd, (bindex, self.imissing), tmp[bindex, self.iknown])
        return fbd


class ADR_Neumann_BounceBack(BounceBackHalfway):
    """``src/darcy.py:394-415``."""

    def __init__(self, indices, gridInfo, precision_policy):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ADR_Neumann_BounceBack"


class ADR_EquilibriumBC(BoundaryCondition):
    """``src/darcy.py:417-466``."""

    def __init__(self, indices, gridInfo, precision_policy, rho, vel=None):
        super().__init__(indices, gridInfo, precision_policy)
        if vel is None:
            self.out = self.precisionPolicy.cast_to_output(np.asarray(rho) * self.lattice.w)
        else:
            self.out = self.precisionPolicy.cast_to_output(self.equilibrium(rho, vel))
        self.name = "ADR_EquilibriumBC"
        self.implementationStep = "PostStreaming"

    def apply(self, fout, fin):
        return self.out
