"""``jax.numpy`` on NumPy: every function returns an ``Array`` (a NumPy array
subclass with JAX's functional ``.at[...]`` updates)."""
import numpy as _np

ndarray = None   # set below (type annotations in the reference name jax.numpy.ndarray)


def _norm_index(idx, shape, clamp):
    """Index tuple with integer-array components normalised the JAX way:
    negative entries count from the end; out-of-range entries are clamped
    (gathers) or replaced by the dimension size (scatters: the pad slot)."""
    if not isinstance(idx, tuple):
        idx = (idx,)
    consumed = sum(1 if not (c is None or c is Ellipsis) else 0 for c in idx)
    consumed += sum(_np.asarray(c).ndim - 1 for c in idx
                    if isinstance(c, (_np.ndarray, list)) and _np.asarray(c).dtype == bool)
    out, dim, padded = [], 0, []
    for c in idx:
        if c is None:
            out.append(c)
            continue
        if c is Ellipsis:
            out.append(c)
            dim += len(shape) - consumed
            continue
        if isinstance(c, (list, _np.ndarray)):
            a = _np.asarray(c)
            if a.dtype == bool:
                out.append(a)
                dim += a.ndim
                continue
            n = shape[dim]
            a = _np.where(a < 0, a + n, a)
            if clamp:
                a = _np.clip(a, 0, n - 1)
            else:
                bad = (a < 0) | (a >= n)
                if _np.any(bad):
                    a = _np.where(bad, n, a)
                    padded.append(dim)
            out.append(a)
        else:
            out.append(c)
        dim += 1
    return tuple(out), padded


class _Update:
    def __init__(self, x, idx):
        self.x, self.idx = x, idx

    def _scatter(self, values, op):
        x = _np.array(self.x, copy=True)
        idx, padded = _norm_index(self.idx, x.shape, clamp=False)
        if padded:
            pad = [(0, 1 if d in padded else 0) for d in range(x.ndim)]
            xp = _np.pad(x, pad)
        else:
            xp = x
        v = _np.asarray(values)
        if op == "set":
            xp[idx] = v.astype(x.dtype, copy=False) if v.dtype != x.dtype else v
        elif op == "add":
            _np.add.at(xp, idx, v)
        elif op == "multiply":
            _np.multiply.at(xp, idx, v)
        elif op == "min":
            _np.minimum.at(xp, idx, v)
        elif op == "max":
            _np.maximum.at(xp, idx, v)
        if padded:
            xp = xp[tuple(slice(0, s) for s in x.shape)]
        return _np.ascontiguousarray(xp).view(Array)

    def set(self, values, **_):
        return self._scatter(values, "set")

    def add(self, values, **_):
        return self._scatter(values, "add")

    def multiply(self, values, **_):
        return self._scatter(values, "multiply")

    def min(self, values, **_):
        return self._scatter(values, "min")

    def max(self, values, **_):
        return self._scatter(values, "max")

    def get(self, **_):
        return self.x[self.idx]


class _At:
    def __init__(self, x):
        self.x = x

    def __getitem__(self, idx):
        return _Update(self.x, idx)


class Array(_np.ndarray):
    """NumPy array with JAX's ``.at`` property and clamping gathers."""

    @property
    def at(self):
        return _At(self)

    def __getitem__(self, idx):
        idx, _ = _norm_index(idx, self.shape, clamp=True)
        return _wrap(_np.ndarray.__getitem__(self, idx))

    # JAX arrays are immutable: augmented assignment rebinds the name to a new
    # array and never changes an array that another name still refers to
    def __iadd__(self, o):
        return _wrap(_np.add(self, o))

    def __isub__(self, o):
        return _wrap(_np.subtract(self, o))

    def __imul__(self, o):
        return _wrap(_np.multiply(self, o))

    def __itruediv__(self, o):
        return _wrap(_np.true_divide(self, o))

    def __ipow__(self, o):
        return _wrap(_np.power(self, o))

    def __setitem__(self, idx, value):
        raise TypeError("JAX arrays are immutable; use x.at[idx].set(value)")

    def block_until_ready(self):
        return self

    @property
    def sharding(self):
        return None


ndarray = Array


def _wrap(r):
    if isinstance(r, _np.ndarray):
        return r.view(Array)
    if isinstance(r, (_np.generic, float, int, bool, complex)):
        return _np.asarray(r).view(Array)
    if isinstance(r, tuple):
        return tuple(_wrap(v) for v in r)
    if isinstance(r, list):
        return [_wrap(v) for v in r]
    return r


def _base(x):
    if isinstance(x, Array):
        return x.view(_np.ndarray)
    if isinstance(x, (list, tuple)):
        return type(x)(_base(v) for v in x)
    return x


def _lift(fn):
    """A NumPy function on plain ndarrays (NumPy's own Python code assigns into
    its intermediate arrays), its results wrapped as ``Array``."""
    def f(*a, **k):
        return _wrap(fn(*[_base(v) for v in a], **{kk: _base(v) for kk, v in k.items()}))
    f.__name__ = getattr(fn, "__name__", "f")
    return f


def array(obj, dtype=None, copy=True, **_):
    return _np.array(obj, dtype=dtype).view(Array)


def asarray(obj, dtype=None, **_):
    return _np.array(obj, dtype=dtype).view(Array)


newaxis = None
float16, float32, float64 = _np.float16, _np.float32, _np.float64
int8, int16, int32, int64 = _np.int8, _np.int16, _np.int32, _np.int64
uint8, uint32 = _np.uint8, _np.uint32
bool_ = _np.bool_
pi = _np.pi
inf, nan = _np.inf, _np.nan
dtype = _np.dtype
linalg = type("linalg", (), {"norm": staticmethod(_lift(_np.linalg.norm))})


def __getattr__(name):
    v = getattr(_np, name)
    return _lift(v) if callable(v) and not isinstance(v, type) else v
