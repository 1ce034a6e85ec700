"""Unit bookkeeping and field utilities (mirror of ``src/utils.py:17-106``)."""
import numpy as np
import torch


class Parameters:
    """``src/utils.py:17-76``: base units plus parameters carrying unit exponents;
    ``get_nondimensional`` divides by the product of the units' powers."""

    def __init__(self, units={}, parameters={}):
        self._units = {}
        self._params = {}
        self.add_units(**units)
        self.add_parameters(**parameters)

    def set_unit(self, name, value):
        if not isinstance(value, float) or value <= 0.0:
            raise TypeError(f"Unit '{name}' must be a positive float.")
        self._units[name] = value

    def add_units(self, **kwargs):
        for k, v in kwargs.items():
            self.set_unit(k, v)

    def set_parameter(self, name, value, unit):
        if not isinstance(unit, dict):
            raise TypeError("unit must be a dict.")
        if not isinstance(value, float):
            raise TypeError("value must be a float.")
        for k, v in unit.items():
            if k not in self._units:
                raise TypeError(f"unit['{k}'] must exist as base unit.")
            if not isinstance(v, int):
                raise TypeError(f"unit['{k}'] must be an int.")
        self._params[name] = (value, unit)

    def add_parameters(self, **kwargs):
        for k, v in kwargs.items():
            self.set_parameter(k, *v)

    def get_unit(self, key):
        return self._units[key]

    def get(self, key):
        return self._params[key][0]

    def get_nondimensional(self, key):
        value, unit = self._params[key]
        for k, v in unit.items():
            value /= self._units[k] ** v
        return value

    def print(self, nondimensional=True):
        print(f"{'Parameter':>20} | {'Unit': ^20} | {'Value'}")
        print('-' * 60)
        for k, v in self._units.items():
            print(f"{k:>20} | {'< UNIT >': ^20} | {v}")
        for k, (v, u) in self._params.items():
            unit = ""
            for uk, uv in u.items():
                if nondimensional:
                    v /= self._units[uk] ** uv
                unit += (" " if len(unit) > 0 else "") + uk + (f"**{uv}" if uv != 1 else "")
            if len(unit) == 0:
                unit = "---"
            print(f"{k:>20} | {unit: ^20} | {v}")


def _keys_cubic(x, a=-0.5):
    x = np.abs(x)
    return np.where(x <= 1, ((a + 2) * x - (a + 3)) * x * x + 1,
                    np.where(x < 2, ((a * x - 5 * a) * x + 8 * a) * x - 4 * a, 0.0))


def _resize_matrix(n_in, n_out):
    """Antialiased Keys-cubic (a=-0.5) resampling weights of a scale-and-translate
    resize with half-pixel centres, the method ``jax.image.resize(..., 'bicubic')``
    uses."""
    scale = n_out / n_in
    ks = max(1.0, 1.0 / scale)          # kernel widened when downsampling (antialias)
    out_c = (np.arange(n_out) + 0.5) / scale - 0.5
    x = np.arange(n_in)
    w = _keys_cubic((x[None, :] - out_c[:, None]) / ks)
    s = w.sum(axis=1, keepdims=True)
    return w / np.where(s == 0, 1, s)


def downsample_field(field, factor, method='bicubic'):
    """``src/utils.py:78-106``: downsample every component by ``factor``."""
    if factor == 1:
        return field
    if method != 'bicubic':
        raise NotImplementedError("only the reference's default 'bicubic' method is provided")
    t = field if isinstance(field, torch.Tensor) else torch.as_tensor(np.asarray(field))
    nx, ny = t.shape[0], t.shape[1]
    mx = torch.as_tensor(_resize_matrix(nx, nx // factor), dtype=t.dtype, device=t.device)
    my = torch.as_tensor(_resize_matrix(ny, ny // factor), dtype=t.dtype, device=t.device)
    return torch.einsum("ax,xyc,by->abc", mx, t, my)
