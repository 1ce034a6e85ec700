"""One-CPU-device stand-in for the parts of ``jax`` the reference imports
(fixture generation only; see README.md beside this package)."""
import functools as _functools

import numpy as _np

from . import numpy  # noqa: F401
from . import lax  # noqa: F401
from . import sharding  # noqa: F401
from . import experimental  # noqa: F401
from . import image  # noqa: F401
from .numpy import Array, _wrap

__version__ = "0.5.3-numpy-standin"


class _Config:
    def __init__(self):
        self.values = {"jax_enable_x64": False}

    def update(self, name, value):
        self.values[name] = value


config = _Config()


def jit(fun=None, static_argnums=(), **kw):
    """Eager call whose non-static NumPy array arguments become ``Array``s, as
    a traced call would see them (jax arrays with ``.at``)."""
    if fun is None:
        return lambda f: jit(f, static_argnums=static_argnums, **kw)
    static = {static_argnums} if isinstance(static_argnums, int) else set(static_argnums)

    def lift(i, a):
        if i not in static and isinstance(a, _np.ndarray) and not isinstance(a, Array):
            return a.view(Array)
        return a

    @_functools.wraps(fun)
    def call(*args, **kwargs):
        args = [lift(i, a) for i, a in enumerate(args)]
        kwargs = {k: lift(-1, v) for k, v in kwargs.items()}
        return fun(*args, **kwargs)
    return call


def vmap(fun, in_axes=0, out_axes=0):
    """Map over one axis of each mapped argument (moved to the front), calling
    ``fun`` per slice and stacking the results along ``out_axes``."""
    def mapped(*args):
        axes = list(in_axes) if isinstance(in_axes, (tuple, list)) else [in_axes] * len(args)
        moved = [None if ax is None else _np.moveaxis(_np.asarray(a), ax, 0) for a, ax in zip(args, axes)]
        n = next(m.shape[0] for m in moved if m is not None)
        outs = [fun(*[_wrap(m[i]) if m is not None else a for a, m in zip(args, moved)]) for i in range(n)]

        def stack(parts, ax):
            return _wrap(_np.stack([_np.asarray(p) for p in parts], axis=ax))
        if isinstance(outs[0], tuple):
            oax = out_axes if isinstance(out_axes, (tuple, list)) else [out_axes] * len(outs[0])
            return tuple(stack(o, ax) for o, ax in zip(zip(*outs), oax))
        return stack(outs, out_axes)
    return mapped


def device_count():
    return 1


def local_device_count():
    return 1


def process_count():
    return 1


def process_index():
    return 0


def devices():
    return ["cpu:0"]


def default_backend():
    return "cpu"


def block_until_ready(x):
    return x


def device_put(x, *_, **__):
    return _wrap(_np.asarray(x))


def tree_map(fn, tree, *rest):
    if isinstance(tree, dict):
        return {k: tree_map(fn, v, *[r[k] for r in rest]) for k, v in tree.items()}
    if isinstance(tree, (list, tuple)):
        return type(tree)(tree_map(fn, v, *[r[i] for r in rest]) for i, v in enumerate(tree))
    return fn(tree, *rest)


class _Distributed:
    @staticmethod
    def initialize(*_, **__):
        return None


distributed = _Distributed()
default_device = None
