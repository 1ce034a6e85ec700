"""Boundary-condition objects (host side), mirror of ``src/boundary_conditions.py``.

These classes keep the reference's constructor signatures, attributes and
preprocessing methods (``create_local_mask_and_normal_arrays``,
``get_boundary_mask``, ``configure``, ``get_normals``, ``get_missing_indices``,
``get_missing_mask``), so user subclasses that override them -- such as the
corner-patched classes of the reference's Terzaghi example -- behave as in the
reference.  ``apply(fout, fin)`` is the reference's per-boundary-cell formula
on NumPy arrays; it is never run in the time loop.  Instead
``bc_compile.compile_rules`` probes it once to turn the ordered BC list into
per-cell affine rules that the CUDA sweeps apply in-kernel.

JAX indexing semantics that the formulas rely on are reproduced by
``_at_set`` / ``_at_add``: duplicate scatter indices -> last write wins for
``set`` and accumulate for ``add``; gathers clamp, scatters drop out-of-range.
"""
import numpy as np


def _bcast_idx(idx):
    return tuple(np.asarray(a).astype(np.int64) for a in np.broadcast_arrays(*[np.asarray(i) for i in idx]))


def _take(arr, idx):
    """JAX gather: indices clamped into range."""
    idx = _bcast_idx(idx)
    return arr[tuple(np.clip(i, 0, arr.shape[d] - 1) for d, i in enumerate(idx))]


def _flat(arr, idx, vals):
    idx = _bcast_idx(idx)
    nd = len(idx)
    vals = np.broadcast_to(np.asarray(vals, dtype=arr.dtype), idx[0].shape + arr.shape[nd:])
    fi = [i.reshape(-1) for i in idx]
    fv = vals.reshape((-1,) + arr.shape[nd:])
    ok = np.logical_and.reduce([(i >= 0) & (i < arr.shape[d]) for d, i in enumerate(fi)])
    return fi, fv, ok, nd


def _at_set(arr, idx, vals):
    """``arr.at[idx].set(vals)`` in place: the last duplicate wins."""
    fi, fv, ok, nd = _flat(arr, idx, vals)
    sel = np.nonzero(ok)[0]
    if sel.size == 0:
        return arr
    lin = np.ravel_multi_index(tuple(i[sel] for i in fi), arr.shape[:nd])
    # walk backwards, keep the first time each target is seen
    _, first_rev = np.unique(lin[::-1], return_index=True)
    keep = sel[::-1][first_rev]
    arr[tuple(i[keep] for i in fi)] = fv[keep]
    return arr


def _at_add(arr, idx, vals):
    """``arr.at[idx].add(vals)`` in place: duplicates accumulate."""
    fi, fv, ok, nd = _flat(arr, idx, vals)
    np.add.at(arr, tuple(i[ok] for i in fi), fv[ok])
    return arr


def grid_mask(nx, ny, lattice, solid_voxels, nz=0):
    """Grid mask of ``src/elasticity.py:460-487`` / ``src/base.py:414-449`` on one
    device: (nx+2, ny+2, [nz+2,] q), True on the one-cell halo (also where the
    domain is periodic) and on solid BC voxels, then streamed."""
    shape = (nx, ny) if lattice.d == 2 else (nx, ny, nz)
    d = len(shape)
    m = np.ones(tuple(n + 2 for n in shape) + (lattice.q,), dtype=bool)
    m[tuple(slice(1, -1) for _ in shape)] = False
    if solid_voxels is not None:
        v = np.asarray(solid_voxels)
        m[tuple(v[:, k] + 1 for k in range(d))] = True
    out = np.empty_like(m)
    for i in range(lattice.q):
        out[..., i] = np.roll(m[..., i], tuple(int(lattice.c[k, i]) for k in range(d)), axis=tuple(range(d)))
    return out


def solid_halo_voxels(bcs):
    lst = [np.array(bc.indices).T for bc in bcs if bc.isSolid]
    return np.unique(np.vstack(lst), axis=0) if lst else None


class PrecisionPolicy:
    """The jmp-policy attributes BC objects read (compute / output dtype)."""

    def __init__(self, compute_dtype, output_dtype):
        self.compute_dtype = compute_dtype
        self.param_dtype = compute_dtype
        self.output_dtype = output_dtype

    def cast_to_compute(self, x):
        if isinstance(x, tuple):
            return tuple(self.cast_to_compute(v) for v in x)
        return None if x is None else np.asarray(x, dtype=self.compute_dtype)

    def cast_to_output(self, x):
        return None if x is None else np.asarray(x, dtype=self.output_dtype)


class BoundaryCondition:
    """``src/boundary_conditions.py:5-349``."""

    def __init__(self, indices, gridInfo, precision_policy):
        self.lattice = gridInfo["lattice"]
        self.nx = gridInfo["nx"]
        self.ny = gridInfo["ny"]
        self.nz = gridInfo["nz"]
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
        """``:87-109`` (one device: indices shifted by the halo width 1)."""
        shifted = np.array(self.indices)
        shifted[0] += 1
        shifted[1:] += 1
        return np.array(grid_mask[tuple(shifted)])

    def configure(self, boundaryMask):
        return

    def prepare_populations(self, fout, fin, implementation_step):
        return fout

    def get_normals(self, boundaryMask):
        """``:155-176``."""
        main_c = self.lattice.c.T[self.lattice.main_indices].astype(np.int64)
        return -np.dot(boundaryMask[..., self.lattice.main_indices], main_c)

    def get_missing_indices(self, boundaryMask):
        """``:178-206`` (zero-padded tables)."""
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

    def _halfway_index_shift(self, boundaryMask):
        """Halfway-BC index shift onto the fluid neighbours of the solid voxels,
        shared by every halfway BC of the reference (``src/elasticity.py:1595-1603``,
        ``src/darcy.py:346-353``, ``src/boundary_conditions.py:499-506``).
        Returns the ``return_index`` array of ``np.unique``."""
        has_fluid = ~boundaryMask[:, self.lattice.opp_indices]
        idx = np.array(self.indices).T
        targets = np.vstack([idx[has_fluid[:, i], :] + self.lattice.c[:, i].astype(np.int64)
                             for i in range(self.lattice.q)])
        uniq, first = np.unique(targets, axis=0, return_index=True)
        self.indices = tuple(uniq.T)
        return first

    def apply(self, fout, fin):
        raise NotImplementedError

    def equilibrium(self, rho, u):
        """``:235-262`` (host NumPy; used by ``ADR_EquilibriumBC``)."""
        dt = np.dtype(self.precisionPolicy.compute_dtype)
        rho, u = np.asarray(rho, dtype=dt), np.asarray(u, dtype=dt)
        c = np.array(self.lattice.c, dtype=dt)
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
        self._halfway_index_shift(boundaryMask)
        if nbd_orig != len(self.indices[0]) and self.vel is not None:
            vel_avg = np.mean(self.vel, axis=0)
            self.vel = np.zeros((len(self.indices[0]), self.lattice.d)) + vel_avg

    def apply(self, fout, fin):
        nbd = len(self.indices[0])
        bindex = np.arange(nbd)[:, None]
        fbd = np.array(_take(fout, self.indices))
        _at_set(fbd, (bindex, self.imissing), _take(fin, self.indices)[bindex, self.iknown])
        if self.vel is not None:
            c = np.array(self.lattice.c, dtype=fbd.dtype)
            cu = 6.0 * self.lattice.w * np.dot(self.vel, c)
            _at_add(fbd, (bindex, self.imissing), -cu[bindex, self.iknown])
        return fbd


class BounceBack(BoundaryCondition):
    """``src/boundary_conditions.py:351-394``: full-way bounce-back, after the
    collision: the wall cell's output is its input reflected, fin[opp]."""

    def __init__(self, indices, gridInfo, precision_policy):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "BounceBackFullway"
        self.implementationStep = "PostCollision"

    def apply(self, fout, fin):
        return np.array(_take(fin, self.indices))[:, self.lattice.opp_indices]


class EquilibriumBC(BoundaryCondition):
    """``src/boundary_conditions.py:549-595``: the populations of the boundary
    cells are set, after streaming, to the equilibrium of (``rho``, ``u``)."""

    def __init__(self, indices, gridInfo, precision_policy, rho, u):
        super().__init__(indices, gridInfo, precision_policy)
        self.out = self.equilibrium(rho, u)
        self.name = "EquilibriumBC"
        self.implementationStep = "PostStreaming"

    def apply(self, fout, fin):
        return self.out


def apply_in_order(bcs, fout, fin, implementation_step=None, names=None):
    """Apply an ordered BC list to full-grid arrays (in place on ``fout``), as
    ``apply_bc`` (``src/elasticity.py:1061-1091``) does for one implementation
    step, or as ``gradient`` (``src/darcy.py:100-103``) does for a name filter."""
    for bc in bcs:
        if implementation_step is not None:
            fout = bc.prepare_populations(fout, fin, implementation_step)
            if bc.implementationStep != implementation_step:
                continue
        elif bc.name not in names:
            continue
        if bc.isDynamic:
            raise NotImplementedError("time-dependent BCs are not on the Biot path")
        _at_set(fout, bc.indices, bc.apply(fout, fin))
    return fout
