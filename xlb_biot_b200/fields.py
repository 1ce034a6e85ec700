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
    several fields with the same geometry.  A three-dimensional grid (nz > 0)
    stores its rows (y, z) as ny * nz rows of one plane, z slowest; users see
    an (nx, ny, nz, c) view."""

    def __init__(self, nx, ny, dtype, device=None, nz=0):
        self.nx, self.ny, self.nz, self.dtype = int(nx), int(ny), int(nz), dtype
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.pitch = pitch_for(nx, dtype)
        self.rows = self.ny * (self.nz if self.nz > 0 else 1)
        self.plane = self.pitch * self.rows

    @property
    def shape(self):
        return (self.nx, self.ny) if self.nz == 0 else (self.nx, self.ny, self.nz)

    def grid(self):
        """The 2-D grid of the kernels: nx columns, all rows (ny, or ny * nz)."""
        return _lib.Grid(self.nx, self.rows, self.pitch, self.plane)

    def grid3(self):
        return _lib.Grid3(self.nx, self.ny, max(self.nz, 1), self.pitch, self.plane)

    def _strides(self):
        return (1, self.pitch) if self.nz == 0 else (1, self.pitch, self.pitch * self.ny)

    def empty(self, c):
        buf = torch.empty(c * self.plane, dtype=self.dtype, device=self.device)
        return buf.as_strided(self.shape + (c,), self._strides() + (self.plane,))

    def zeros(self, c):
        t = self.empty(c)
        buf_of(t).zero_()
        return t

    def conforms(self, t, c=None):
        nd = len(self.shape)
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == self.dtype and t.dim() == nd + 1
                and tuple(t.shape[:nd]) == self.shape and (c is None or t.shape[nd] == c)
                and t.device == self.device):
            return False
        st = self._strides()
        for k in range(nd):
            if t.shape[k] > 1 and t.stride(k) != st[k]:
                return False
        return t.shape[nd] == 1 or t.stride(nd) == self.plane

    def field(self, x, c=None):
        """A conforming tensor with the values of ``x`` (numpy array, torch tensor
        or scalar broadcast to ``shape + (c,)``); no copy if ``x`` conforms."""
        if x is None:
            return None
        if self.conforms(x, c):
            return x
        if isinstance(x, torch.Tensor):
            src = x.to(device=self.device, dtype=self.dtype)
        else:
            src = torch.as_tensor(np.asarray(x), device=self.device).to(self.dtype)
        nd = len(self.shape)
        if src.dim() == nd:
            src = src[..., None]
        if c is None:
            c = src.shape[-1] if src.dim() == nd + 1 else 1
        out = self.empty(c)
        out.copy_(torch.broadcast_to(src, self.shape + (c,)))
        return out


def buf_of(t):
    """The flat plane buffer behind a conforming field view."""
    c = t.shape[-1]
    if c > 1:
        n = c * t.stride(-1)
    else:
        n = t.shape[-2] * t.stride(-2)
    return t.as_strided((n,), (1,))
