"""JAX indexing semantics restated in NumPy (oracle only).

``jnp`` differs from NumPy in three places the reference's boundary conditions
depend on (``src/boundary_conditions.py:178-206`` pads ``imissing/iknown`` with
index 0, so scatters regularly carry duplicate indices):

* scatter-set with duplicates  -> last update in row-major order wins;
* scatter-add with duplicates  -> every update accumulates (``np.add.at``);
* gather out of range          -> index clamped to the valid range;
* scatter out of range         -> update dropped.
"""
import numpy as np


def _broadcast_index(idx):
    arrs = np.broadcast_arrays(*[np.asarray(i) for i in idx])
    return tuple(a.astype(np.int64) for a in arrs)


def gather(arr, idx):
    """``arr[idx]`` for the leading ``len(idx)`` axes with JAX clamping."""
    idx = _broadcast_index(idx)
    clipped = tuple(np.clip(i, 0, arr.shape[d] - 1) for d, i in enumerate(idx))
    return arr[clipped]


def scatter_set(arr, idx, vals):
    """``arr.at[idx].set(vals)`` (returns a new array).  Last duplicate wins,
    out-of-range updates are dropped."""
    out = np.array(arr, copy=True)
    idx = _broadcast_index(idx)
    nd = len(idx)
    vals = np.broadcast_to(np.asarray(vals, dtype=out.dtype),
                           idx[0].shape + out.shape[nd:])
    flat_idx = [i.reshape(-1) for i in idx]
    flat_vals = vals.reshape((-1,) + out.shape[nd:])
    ok = np.ones(flat_idx[0].shape, dtype=bool)
    for d, i in enumerate(flat_idx):
        ok &= (i >= 0) & (i < out.shape[d])
    lin = np.ravel_multi_index(tuple(np.where(ok, i, 0) for i in flat_idx), out.shape[:nd])
    sel = np.nonzero(ok)[0]
    # keep the last occurrence of every target
    rev = sel[::-1]
    _, first_in_rev = np.unique(lin[rev], return_index=True)
    keep = rev[first_in_rev]
    tgt = tuple(i[keep] for i in flat_idx)
    out[tgt] = flat_vals[keep]
    return out


def scatter_add(arr, idx, vals):
    """``arr.at[idx].add(vals)`` (returns a new array).  Duplicates accumulate,
    out-of-range updates are dropped."""
    out = np.array(arr, copy=True)
    idx = _broadcast_index(idx)
    nd = len(idx)
    vals = np.broadcast_to(np.asarray(vals, dtype=out.dtype),
                           idx[0].shape + out.shape[nd:])
    flat_idx = [i.reshape(-1) for i in idx]
    flat_vals = vals.reshape((-1,) + out.shape[nd:])
    ok = np.ones(flat_idx[0].shape, dtype=bool)
    for d, i in enumerate(flat_idx):
        ok &= (i >= 0) & (i < out.shape[d])
    np.add.at(out, tuple(i[ok] for i in flat_idx), flat_vals[ok])
    return out


def bool_mask_set(arr, mask, vals):
    """``arr.at[mask].set(vals)`` for a boolean mask (row-major order)."""
    out = np.array(arr, copy=True)
    out[mask] = vals
    return out
