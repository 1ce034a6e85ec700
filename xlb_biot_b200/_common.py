"""Helpers shared by the solver classes: precision policy, parameter tables,
host copies for the ``output_data`` hooks."""
import numpy as np
import torch

from . import _lib
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
    """The precision policy of ``precision`` (``src/elasticity.py:606-629``).
    Supported: 'f64/f64', 'f32/f32' and 'f64/f32' (FP32 storage, FP64
    arithmetic in every collide-and-stream sweep with FP64 boundary constants;
    the auxiliary kernels -- moments, gradients, transfers -- compute in the
    FP32 storage type).  Half-precision storage is not provided."""
    compute, stored = set_precisions(precision)
    if stored == np.float16 or compute == np.float16:
        raise NotImplementedError(f"precision {precision!r}: half-precision storage is not supported by the "
                                  "CUDA kernels; use 'f32/f32', 'f64/f32' or 'f64/f64'")
    return PrecisionPolicy(compute, stored)


def storage_and_sweep_dtypes(policy):
    """(storage torch dtype, whether sweeps compute in FP64 on FP32 storage)."""
    storage = torch.float64 if np.dtype(policy.output_dtype) == np.float64 else torch.float32
    acc64 = np.dtype(policy.compute_dtype) == np.float64 and storage == torch.float32
    return storage, acc64


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


def require_finite(value, what, iteration):
    """Raise ``NonFiniteError`` (XLBB_ENONFINITE) when a convergence measure
    (scalar or per-instance array) holds NaN or Inf."""
    v = np.asarray(value, dtype=np.float64)
    if not np.all(np.isfinite(v)):
        where = "" if v.ndim == 0 else f" (instances {np.flatnonzero(~np.isfinite(v))[:8].tolist()})"
        raise _lib.NonFiniteError(f"XLBB_ENONFINITE: {what} is not finite after {iteration} iterations{where}: "
                                  "the iteration diverged or a field holds NaN/Inf")


def iterate_to_tolerance(advance, tol, max_iters, stall_checks=None, what="relative residual"):
    """Host driver of the pseudo-time and V-cycle loops.  ``advance()`` runs the
    next batch of iterations on the device and returns ``(iterations run,
    relative residual)``.  Stops when the residual is below ``tol``, when
    ``max_iters`` iterations have run, or -- with ``stall_checks`` -- when the
    residual has not fallen by 1 % for that many checks (the rounding floor of
    the storage precision).  A NaN or Inf residual raises ``NonFiniteError``
    at once.  Returns ``(iterations, relative residual, stalled)``."""
    it, rel = 0, 1.0
    best, since_best = np.inf, 0
    while it < max_iters:
        n, rel = advance()
        it += n
        require_finite(rel, what, it)
        if rel < tol:
            return it, rel, False
        if stall_checks:
            if rel < 0.99 * best:
                best, since_best = rel, 0
            else:
                since_best += 1
                if since_best >= stall_checks:
                    return it, rel, True
    return it, rel, False
