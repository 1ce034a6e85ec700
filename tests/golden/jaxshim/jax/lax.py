"""``jax.lax`` pieces the reference uses, on NumPy."""
import numpy as _np

from .numpy import _wrap


def with_sharding_constraint(x, sharding):
    return x


def ppermute(x, axis_name, perm):
    """A ring permutation over one device returns its input."""
    if any(a != b for a, b in perm):
        raise NotImplementedError("ppermute across devices: the stand-in has one device")
    return x


def conv_dimension_numbers(lhs_shape, rhs_shape, specs):
    return tuple(specs)


def conv_general_dilated(lhs, rhs, window_strides, padding, lhs_dilation=None, rhs_dilation=None,
                         dimension_numbers=None, **_):
    """XLA convolution (cross-correlation, no kernel flip) for two spatial
    dimensions: lhs dilated by inserting ``d - 1`` zeros between elements,
    padded, correlated with the (dilated) kernel at the window strides."""
    lhs_spec, rhs_spec, out_spec = dimension_numbers
    lhs, rhs = _np.asarray(lhs), _np.asarray(rhs)
    sp = [c for c in lhs_spec if c not in "NC"]
    x = _np.transpose(lhs, [lhs_spec.index(c) for c in "NC" + "".join(sp)])          # N, C, s0, s1
    k = _np.transpose(rhs, [rhs_spec.index(c) for c in "OI" + "".join(c for c in rhs_spec if c not in "OI")])
    nd = x.ndim - 2
    lhs_dilation = tuple(lhs_dilation or (1,) * nd)
    rhs_dilation = tuple(rhs_dilation or (1,) * nd)
    if any(d != 1 for d in lhs_dilation):
        shape = list(x.shape[:2]) + [(s - 1) * d + 1 for s, d in zip(x.shape[2:], lhs_dilation)]
        xd = _np.zeros(shape, dtype=x.dtype)
        xd[(slice(None), slice(None)) + tuple(slice(None, None, d) for d in lhs_dilation)] = x
        x = xd
    if any(d != 1 for d in rhs_dilation):
        shape = list(k.shape[:2]) + [(s - 1) * d + 1 for s, d in zip(k.shape[2:], rhs_dilation)]
        kd = _np.zeros(shape, dtype=k.dtype)
        kd[(slice(None), slice(None)) + tuple(slice(None, None, d) for d in rhs_dilation)] = k
        k = kd
    if isinstance(padding, str):
        if padding != "VALID":
            raise NotImplementedError(padding)
        padding = [(0, 0)] * nd
    x = _np.pad(x, [(0, 0), (0, 0)] + [tuple(p) for p in padding])
    ks = k.shape[2:]
    outs = [(x.shape[2 + i] - ks[i]) // window_strides[i] + 1 for i in range(nd)]
    out = _np.zeros((x.shape[0], k.shape[0]) + tuple(outs), dtype=_np.result_type(x, k))
    for taps in _np.ndindex(*ks):
        win = x[(slice(None), slice(None)) + tuple(
            slice(t, t + (o - 1) * s + 1, s) for t, o, s in zip(taps, outs, window_strides))]
        out += _np.einsum("nc...,oc->no...", win, k[(slice(None), slice(None)) + taps])
    # N, O, spatial -> out_spec (out_spec uses N for batch, C for feature)
    cur = "NC" + "".join(sp)
    return _wrap(_np.transpose(out, [cur.index(c) for c in out_spec]))
