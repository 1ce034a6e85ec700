"""Fluid BGK (D2Q9, D3Q19, D3Q27) and KBC (D2Q9) collision models (oracle) — TEST INFRASTRUCTURE ONLY.

Restates ``src/models.py:9-154`` (``BGKSim``, ``KBCSim``, the D2Q9 shear
decomposition) on the ``LBMBase`` pieces they use (``src/base.py:351-372``
set-up, ``:528-559`` initial populations, ``:686-772`` equilibrium and
macroscopic fields, ``:809-846`` step, ``:848-948`` run loop) and the
``BounceBack`` / ``EquilibriumBC`` conditions of
``src/boundary_conditions.py:351-394,549-595`` used by
``examples/performance/MLUPS2d.py``.
"""
import numpy as np

from . import jaxsem
from .boundary_conditions import BoundaryCondition, apply_bc_list, create_grid_mask, solid_voxels, stream
from .lattice import Policy


class BounceBack(BoundaryCondition):
    """``src/boundary_conditions.py:351-394``: fin[indices][..., opp] after collision."""

    def __init__(self, indices, gridInfo, precision_policy):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "BounceBackFullway"
        self.implementationStep = "PostCollision"

    def apply(self, fout, fin):
        return jaxsem.gather(fin, self.indices)[..., self.lattice.opp_indices]


class EquilibriumBC(BoundaryCondition):
    """``src/boundary_conditions.py:549-595``: equilibrium of (rho, u) after streaming."""

    def __init__(self, indices, gridInfo, precision_policy, rho, u):
        super().__init__(indices, gridInfo, precision_policy)
        self.out = self.precisionPolicy.cast_to_output(self.equilibrium(rho, u))
        self.name = "EquilibriumBC"
        self.implementationStep = "PostStreaming"

    def apply(self, fout, fin):
        return self.out


class _FluidBase:
    """``src/base.py:30-146`` (one device; two or three dimensions)."""

    def __init__(self, **kwargs):
        self.omega = kwargs.get("omega")
        self.nx, self.ny, self.nz = kwargs.get("nx"), kwargs.get("ny"), kwargs.get("nz")
        self.precision = kwargs.get("precision")
        self.precisionPolicy = Policy(self.precision)
        self.lattice = kwargs.get("lattice")
        self.c, self.q, self.w, self.dim = self.lattice.c, self.lattice.q, self.lattice.w, self.lattice.d
        self.gridInfo = {"nx": self.nx, "ny": self.ny, "nz": self.nz, "dim": self.dim, "lattice": self.lattice}
        nx, ny, nz = self.nx, self.ny, self.nz
        if self.dim == 2:            # src/base.py:451-470
            self.boundingBoxIndices = {
                "bottom": np.array([[i, 0] for i in range(nx)], dtype=int),
                "top": np.array([[i, ny - 1] for i in range(nx)], dtype=int),
                "left": np.array([[0, i] for i in range(ny)], dtype=int),
                "right": np.array([[nx - 1, i] for i in range(ny)], dtype=int)}
        else:                        # src/base.py:472-484
            self.boundingBoxIndices = {
                "bottom": np.array([[i, j, 0] for i in range(nx) for j in range(ny)], dtype=int),
                "top": np.array([[i, j, nz - 1] for i in range(nx) for j in range(ny)], dtype=int),
                "left": np.array([[0, j, k] for j in range(ny) for k in range(nz)], dtype=int),
                "right": np.array([[nx - 1, j, k] for j in range(ny) for k in range(nz)], dtype=int),
                "front": np.array([[i, 0, k] for i in range(nx) for k in range(nz)], dtype=int),
                "back": np.array([[i, ny - 1, k] for i in range(nx) for k in range(nz)], dtype=int)}
        self.BCs = []
        self.set_boundary_conditions()
        grid_mask = create_grid_mask(nx, ny, self.lattice, solid_voxels(self.BCs), nz)
        for bc in self.BCs:
            bc.create_local_mask_and_normal_arrays(grid_mask)

    def set_boundary_conditions(self):
        pass

    def initialize_macroscopic_fields(self):
        return None, None

    def assign_fields_sharded(self):
        """``src/base.py:528-559``."""
        rho0, u0 = self.initialize_macroscopic_fields()
        if rho0 is None or u0 is None:
            shape = (self.nx, self.ny) if self.dim == 2 else (self.nx, self.ny, self.nz)
            return np.broadcast_to(self.w.astype(self.precisionPolicy.output_dtype), shape + (self.q,)).copy()
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

    def update_macroscopic(self, f):
        """``src/base.py:748-772``."""
        rho = np.sum(f, axis=-1, keepdims=True)
        c = np.array(self.c, dtype=self.precisionPolicy.compute_dtype).T
        return rho, np.dot(f, c) / rho

    def step(self, f_poststreaming, timestep, return_fpost=False):
        """``src/base.py:809-846``."""
        f_postcollision = self.collision(f_poststreaming)
        f_postcollision = apply_bc_list(self.BCs, f_postcollision, f_poststreaming, "PostCollision")
        f_new = stream(f_postcollision, self.c)
        f_new = apply_bc_list(self.BCs, f_new, f_postcollision, "PostStreaming")
        return (f_new, f_postcollision) if return_fpost else (f_new, None)

    def run(self, t_max):
        """``src/base.py:848-948`` without I/O: t_max + 1 steps."""
        f = self.assign_fields_sharded()
        for timestep in range(0, t_max + 1):
            f, _ = self.step(f, timestep)
        return f


class BGKSim(_FluidBase):
    """``src/models.py:9-34``."""

    def collision(self, f):
        f = self.precisionPolicy.cast_to_compute(f)
        rho, u = self.update_macroscopic(f)
        feq = self.equilibrium(rho, u, cast_output=False)
        fout = f - self.omega * (f - feq)
        return self.precisionPolicy.cast_to_output(fout)


class KBCSim(_FluidBase):
    """``src/models.py:36-72,115-214`` (D2Q9 and D3Q27)."""

    def __init__(self, **kwargs):
        # src/models.py:42-45
        if kwargs.get("lattice").name != "D3Q27" and kwargs.get("nz") > 0:
            raise ValueError("KBC collision operator in 3D must only be used with D3Q27 lattice.")
        super().__init__(**kwargs)

    def momentum_flux(self, fneq):
        """``src/base.py:727-746``: fneq . cc, cc the products c_a c_b (a <= b,
        row-major: xx, xy[, xz], yy[, yz, zz]) of ``src/lattice.py:184-210``."""
        c = np.array(self.c, dtype=fneq.dtype)
        d = c.shape[0]
        cc = np.stack([c[a] * c[b] for a in range(d) for b in range(a, d)], axis=1)
        return np.dot(fneq, cc)

    def fdecompose_shear_d3q27(self, fneq):
        """``src/models.py:156-214``: with Pi = (xx, xy, xz, yy, yz, zz),
        N_xz = Pi_xx - Pi_zz and N_yz = Pi_yy - Pi_zz, the axis directions get
        (2 N_xz - N_yz) / 6 (x), (2 N_yz - N_xz) / 6 (y), -(N_xz + N_yz) / 6 (z),
        the face diagonals +-Pi_ab / 4 by the sign of c_a c_b, the rest and the
        corners zero."""
        Pi = self.momentum_flux(fneq)
        nxz = Pi[..., 0] - Pi[..., 5]
        nyz = Pi[..., 3] - Pi[..., 5]
        s = np.zeros_like(fneq)
        s[..., 9] = (2.0 * nxz - nyz) / 6.0
        s[..., 18] = (2.0 * nxz - nyz) / 6.0
        s[..., 3] = (-nxz + 2.0 * nyz) / 6.0
        s[..., 6] = (-nxz + 2.0 * nyz) / 6.0
        s[..., 1] = (-nxz - nyz) / 6.0
        s[..., 2] = (-nxz - nyz) / 6.0
        for i, j, comp in ((12, 24, 1), (10, 20, 2), (8, 4, 4)):      # c_a c_b = +1
            s[..., i] = Pi[..., comp] / 4.0
            s[..., j] = Pi[..., comp] / 4.0
        for i, j, comp in ((21, 15, 1), (19, 11, 2), (7, 5, 4)):      # c_a c_b = -1
            s[..., i] = -Pi[..., comp] / 4.0
            s[..., j] = -Pi[..., comp] / 4.0
        return s

    def fdecompose_shear_d2q9(self, fneq):
        """``src/models.py:127-154``; momentum flux ``fneq . cc`` with
        cc = (cx cx, cx cy, cy cy) (``src/base.py:727-746``, ``src/lattice.py:184-210``)."""
        c = np.array(self.c, dtype=fneq.dtype)
        cc = np.stack([c[0] * c[0], c[0] * c[1], c[1] * c[1]], axis=1)
        Pi = np.dot(fneq, cc)
        N = Pi[..., 0] - Pi[..., 2]
        s = np.zeros_like(fneq)
        s[..., 6] = N
        s[..., 3] = N
        s[..., 2] = -N
        s[..., 1] = -N
        s[..., 8] = Pi[..., 1]
        s[..., 4] = -Pi[..., 1]
        s[..., 5] = -Pi[..., 1]
        s[..., 7] = Pi[..., 1]
        return s

    def collision(self, f):
        f = self.precisionPolicy.cast_to_compute(f)
        tiny = 1e-32
        beta = self.omega * 0.5
        rho, u = self.update_macroscopic(f)
        feq = self.equilibrium(rho, u, cast_output=False)
        fneq = f - feq
        if self.dim == 2:
            deltaS = self.fdecompose_shear_d2q9(fneq) * rho / 4.0
        else:
            deltaS = self.fdecompose_shear_d3q27(fneq) * rho
        deltaH = fneq - deltaS
        invBeta = 1.0 / beta
        gamma = invBeta - (2.0 - invBeta) * np.sum(deltaS * deltaH / feq, axis=-1) / (
            tiny + np.sum(deltaH * deltaH / feq, axis=-1))
        fout = f - beta * (2.0 * deltaS + gamma[..., None] * deltaH)
        return self.precisionPolicy.cast_to_output(fout)
