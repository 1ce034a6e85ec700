"""Helpers shared by the solver classes: precision policy, parameter tables,
host copies for the ``output_data`` hooks."""
import numpy as np
import torch

from .boundary_conditions import PrecisionPolicy

_PRECISIONS = {
    "f64/f64": (np.float64, np.float64),
    "f32/f32": (np.float32, np.float32),
    "f32/f16": (np.float32, np.float16),
    "f16/f16": (np.float16, np.float16),
    "f64/f32": (np.float64, np.float32),
    "f64/f16": (np.float64, np.float16),
}


def set_precisions(precision):
    """``src/elasticity.py:606-629``: unknown strings fall back to f32/f32."""
    return _PRECISIONS.get(precision, (np.float32, np.float32))


def make_policy(precision):
    compute, stored = set_precisions(precision)
    if compute != stored:
        raise NotImplementedError(
            f"precision {precision!r}: the CUDA kernels compute in their storage type; "
            "use 'f32/f32' or 'f64/f64'")
    if compute == np.float16:
        raise NotImplementedError("precision 'f16/f16' is not supported by the CUDA kernels")
    return PrecisionPolicy(compute, stored)


def print_parameters(obj, attrs, names):
    """Parameter table of ``show_simulation_parameters`` (``src/elasticity.py:356-394``)."""
    print(f"**** Simulation Parameters for {obj.__class__.__name__} ****")
    print(f"{'Parameter':>30} | Value")
    print("-" * 50)
    for a in attrs:
        print(f"{names.get(a, a):>30} | {getattr(obj, a, 'Attribute not set')}")


def host(x):
    """Device field -> NumPy array (the reference hands ``output_data`` host
    arrays gathered with ``process_allgather``)."""
    if x is None:
        return None
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def gathered(x):
    """``process_allgather`` of one process: a leading axis of length 1."""
    h = host(x)
    return None if h is None else h[None]
