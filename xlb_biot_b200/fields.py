"""Device fields in the kernels' structure-of-arrays layout.

A field of the reference's shape ``(nx, ny, c)`` lives in one CUDA buffer of
``c`` planes, each plane ``ny`` rows of ``pitch`` elements with x fastest.
Users see a strided tensor view of the reference's shape, so indexing such as
``f[x, y, i]`` means exactly what it means for the JAX arrays of the reference,
while the kernels stream whole rows with coalesced loads.
"""
import numpy as np
import torch

from . import _lib

_NP2TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
             np.dtype(np.float16): torch.float16}


def torch_dtype(dt):
    """Map a numpy / torch / jnp-like dtype (or its name) to a torch dtype."""
    if isinstance(dt, torch.dtype):
        return dt
    if isinstance(dt, str):
        dt = np.dtype(dt)
    try:
        return _NP2TORCH[np.dtype(dt)]
    except (TypeError, KeyError):
        raise TypeError(f"unsupported dtype {dt!r}")


def pitch_for(nx, dtype):
    """Row pitch: 16-byte aligned rows (4 FP32 / 2 FP64 elements)."""
    align = max(1, 16 // torch.empty((), dtype=dtype).element_size())
    return (nx + align - 1) // align * align


class Layout:
    """Pitch/plane of all fields of one grid, so that one kernel launch can take
    several fields with the same geometry."""

    def __init__(self, nx, ny, dtype, device=None):
        self.nx, self.ny, self.dtype = int(nx), int(ny), dtype
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.pitch = pitch_for(nx, dtype)
        self.plane = self.pitch * self.ny

    def grid(self):
        return _lib.Grid(self.nx, self.ny, self.pitch, self.plane)

    def empty(self, c):
        buf = torch.empty(c * self.plane, dtype=self.dtype, device=self.device)
        return buf.as_strided((self.nx, self.ny, c), (1, self.pitch, self.plane))

    def zeros(self, c):
        t = self.empty(c)
        buf_of(t).zero_()
        return t

    def conforms(self, t, c=None):
        return (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == self.dtype and t.dim() == 3
                and t.shape[0] == self.nx and t.shape[1] == self.ny and (c is None or t.shape[2] == c)
                and t.stride(0) == 1 and (self.ny == 1 or t.stride(1) == self.pitch)
                and (t.shape[2] == 1 or t.stride(2) == self.plane)
                and t.device == self.device)

    def field(self, x, c=None):
        """A conforming tensor with the values of ``x`` (numpy array, torch tensor
        or scalar broadcast to ``(nx, ny, c)``); no copy if ``x`` conforms."""
        if x is None:
            return None
        if self.conforms(x, c):
            return x
        if isinstance(x, torch.Tensor):
            src = x.to(device=self.device, dtype=self.dtype)
        else:
            src = torch.as_tensor(np.asarray(x), device=self.device).to(self.dtype)
        if src.dim() == 2:
            src = src[..., None]
        if c is None:
            c = src.shape[-1] if src.dim() == 3 else 1
        out = self.empty(c)
        out.copy_(torch.broadcast_to(src, (self.nx, self.ny, c)))
        return out


def buf_of(t):
    """The flat plane buffer behind a conforming field view."""
    return t.as_strided((t.shape[2] * t.stride(2) if t.shape[2] > 1 else t.shape[1] * t.stride(1),), (1,))
