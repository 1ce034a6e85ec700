"""Boundary-condition base and grid mask (oracle).

Restates ``src/boundary_conditions.py:5-233`` (base class), ``:452-547``
(``BounceBackHalfway``) and the grid-mask construction of
``src/elasticity.py:460-499`` / ``src/base.py:414-449`` for one device
(halo width 1 in x and y).
"""
import numpy as np

from . import jaxsem


def stream(f, c):
    """Periodic pull streaming ``f_i(x) <- f_i(x - c_i)`` via ``roll``
    (``src/elasticity.py:768-803``, ``src/base.py:649-683``).  On one device the
    ppermute halo swap of ``streaming_m`` (``:738-766``) is the identity."""
    d = c.shape[0]
    out = np.empty_like(f)
    for i in range(f.shape[-1]):
        out[..., i] = np.roll(f[..., i], tuple(int(c[k, i]) for k in range(d)), axis=tuple(range(d)))
    return out


def create_grid_mask(nx, ny, lattice, solid_halo_voxels, nz=0):
    """``src/elasticity.py:460-487`` / ``src/base.py:414-449``: a (nx+2, ny+2,
    [nz+2,] q) boolean mask, True on the one-cell halo (even for periodic
    sides) and on solid BC voxels, streamed."""
    hw = 1
    shape = (nx, ny) if lattice.d == 2 else (nx, ny, nz)
    m = np.ones(tuple(n + 2 * hw for n in shape) + (lattice.q,), dtype=bool)
    m[tuple(slice(hw, -hw) for _ in shape)] = False
    if solid_halo_voxels is not None:
        v = np.asarray(solid_halo_voxels)
        m[tuple(v[:, k] + hw for k in range(len(shape)))] = True
    return stream(m, lattice.c)


def solid_voxels(bcs):
    """``src/elasticity.py:407-408``: unique indices of all solid BCs."""
    lst = [np.array(bc.indices).T for bc in bcs if bc.isSolid]
    return np.unique(np.vstack(lst), axis=0) if lst else None


class BoundaryCondition:
    """``src/boundary_conditions.py:5-349``."""

    def __init__(self, indices, gridInfo, precision_policy):
        self.lattice = gridInfo["lattice"]
        self.nx, self.ny, self.nz = gridInfo["nx"], gridInfo["ny"], gridInfo["nz"]
        self.dim = gridInfo["dim"]
        self.precisionPolicy = precision_policy
        self.indices = indices
        self.name = None
        self.isSolid = False
        self.isDynamic = False
        self.needsExtraConfiguration = False
        self.implementationStep = "PostStreaming"

    def create_local_mask_and_normal_arrays(self, grid_mask):
        """``:55-85``."""
        if self.needsExtraConfiguration:
            self.configure(self.get_boundary_mask(grid_mask))
            self.needsExtraConfiguration = False
        boundaryMask = self.get_boundary_mask(grid_mask)
        self.normals = self.get_normals(boundaryMask)
        self.imissing, self.iknown = self.get_missing_indices(boundaryMask)
        self.imissingMask, self.iknownMask, self.imiddleMask = self.get_missing_mask(boundaryMask)

    def get_boundary_mask(self, grid_mask):
        """``:87-109`` (device_count() == 1)."""
        s = np.array(self.indices)
        s[0] += 1
        s[1:] += 1
        return np.array(grid_mask[tuple(s)])

    def configure(self, boundaryMask):
        return

    def prepare_populations(self, fout, fin, implementation_step):
        return fout

    def get_normals(self, boundaryMask):
        """``:155-176``."""
        main_c = self.lattice.c.T[self.lattice.main_indices].astype(np.int64)
        m = boundaryMask[..., self.lattice.main_indices]
        return -np.dot(m, main_c)

    def get_missing_indices(self, boundaryMask):
        """``:178-206``: zero-padded missing/known direction tables."""
        nbd = len(self.indices[0])
        imissing = np.vstack([np.arange(self.lattice.q, dtype="uint8")] * nbd)
        iknown = np.vstack([self.lattice.opp_indices] * nbd)
        imissing[~boundaryMask] = 0
        iknown[~boundaryMask] = 0
        return imissing, iknown

    def get_missing_mask(self, boundaryMask):
        """``:208-233``."""
        imissingMask = boundaryMask
        iknownMask = imissingMask[:, self.lattice.opp_indices]
        imiddleMask = ~(imissingMask | iknownMask)
        return imissingMask, iknownMask, imiddleMask

    def halfway_shift(self, boundaryMask):
        """Index shift of the halfway BCs to the fluid neighbours of the solid
        voxels (``src/elasticity.py:1595-1603``, ``src/darcy.py:346-353``,
        ``src/boundary_conditions.py:499-506``).  Returns (new_idx, array_indices)."""
        hasFluidNeighbour = ~boundaryMask[:, self.lattice.opp_indices]
        idx = np.array(self.indices).T
        trg = [idx[hasFluidNeighbour[:, i], :] + self.lattice.c[:, i].astype(np.int64)
               for i in range(self.lattice.q)]
        new, first = np.unique(np.vstack(trg), axis=0, return_index=True)
        self.indices = tuple(new.T)
        return new, first

    def apply(self, fout, fin):
        raise NotImplementedError

    def equilibrium(self, rho, u):
        """``:235-262``."""
        rho, u = self.precisionPolicy.cast_to_compute((rho, u))
        c = np.array(self.lattice.c, dtype=self.precisionPolicy.compute_dtype)
        cu = 3.0 * np.dot(u, c)
        usqr = 1.5 * np.sum(u ** 2, axis=-1, keepdims=True)
        return rho * self.lattice.w * (1.0 + 1.0 * cu + 0.5 * cu ** 2 - usqr)


class BounceBackHalfway(BoundaryCondition):
    """``src/boundary_conditions.py:452-547``."""

    def __init__(self, indices, gridInfo, precision_policy, vel=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "BounceBackHalfway"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.vel = vel

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        new, _ = self.halfway_shift(boundaryMask)
        if nbd_orig != len(self.indices[0]) and self.vel is not None:
            vel_avg = np.mean(self.vel, axis=0)
            self.vel = np.zeros(new.shape, dtype=self.precisionPolicy.compute_dtype) + vel_avg

    def impose_boundary_vel(self, fbd, bindex):
        c = np.array(self.lattice.c, dtype=self.precisionPolicy.compute_dtype)
        cu = 6.0 * self.lattice.w * np.dot(self.vel, c)
        return jaxsem.scatter_add(fbd, (bindex, self.imissing), -cu[bindex, self.iknown])

    def apply(self, fout, fin):
        nbd = len(self.indices[0])
        bindex = np.arange(nbd)[:, None]
        fbd = jaxsem.gather(fout, self.indices)
        fin_bd = jaxsem.gather(fin, self.indices)
        fbd = jaxsem.scatter_set(fbd, (bindex, self.imissing), fin_bd[bindex, self.iknown])
        if self.vel is not None:
            fbd = self.impose_boundary_vel(fbd, bindex)
        return fbd


def apply_bc_list(bcs, fout, fin, implementation_step):
    """``src/elasticity.py:1061-1091`` / ``src/base.py:776-806``."""
    for bc in bcs:
        fout = bc.prepare_populations(fout, fin, implementation_step)
        if bc.implementationStep == implementation_step:
            if bc.isDynamic:
                raise NotImplementedError("dynamic BCs are not on the Biot path")
            fout = jaxsem.scatter_set(fout, bc.indices, bc.apply(fout, fin))
    return fout
