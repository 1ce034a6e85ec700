"""``jmp.Policy``: cast floating-point leaves to the compute / param / output dtype."""
import numpy as _np

from jax.numpy import _wrap


def _cast(tree, dtype):
    if isinstance(tree, (list, tuple)):
        return type(tree)(_cast(v, dtype) for v in tree)
    if isinstance(tree, dict):
        return {k: _cast(v, dtype) for k, v in tree.items()}
    if tree is None:
        return None
    a = _np.asarray(tree)
    if _np.issubdtype(a.dtype, _np.floating):
        return _wrap(a.astype(dtype))
    return tree


class Policy:
    def __init__(self, param_dtype, compute_dtype, output_dtype):
        self.param_dtype, self.compute_dtype, self.output_dtype = param_dtype, compute_dtype, output_dtype

    def cast_to_compute(self, x):
        return _cast(x, self.compute_dtype)

    def cast_to_param(self, x):
        return _cast(x, self.param_dtype)

    def cast_to_output(self, x):
        return _cast(x, self.output_dtype)
