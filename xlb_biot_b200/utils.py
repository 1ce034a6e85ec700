"""Unit bookkeeping, field utilities and VTK output (mirror of
``src/utils.py:17-106,144-196,243-304``)."""
import os
import time

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


def results_filename(output_dir, E, nu, K, alpha, nx, ne, levels, coupling, alternative_gradient=False):
    """Result file of one run of the convergence sweeps, named as
    ``examples/poroelasticity/periodic.py:217`` names it."""
    return os.path.join(output_dir, f"error_E{E:.3f}_nu{nu:.3f}_K{K:.3f}_a{alpha:.3f}_nx{nx:03d}_ne{ne:03d}"
                                    f"_l{levels:03d}_{coupling}{'_altgrad' if alternative_gradient else ''}.npz")


def cached_results(filename, compute):
    """``examples/poroelasticity/periodic.py:218-259``: the arrays of an earlier
    run loaded from ``filename`` (``.npz``), or -- when the file is missing or
    unreadable -- ``compute()`` (a dict of arrays) run and saved compressed.
    Returns a dict of NumPy arrays either way."""
    try:
        with np.load(filename) as data:
            return {k: data[k] for k in data.files}
    except Exception:
        pass
    data = {k: np.asarray(v) for k, v in compute().items()}
    os.makedirs(os.path.dirname(os.path.abspath(filename)), exist_ok=True)
    np.savez_compressed(filename, **data)
    return data


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


# ---------------------------------------------------------------------------
# Legacy-VTK output.  The reference writes these files through pyvista
# (``pv.ImageData(...).save(name, binary=True)``), which is not a dependency
# here: the same file layout is written directly (legacy VTK, binary,
# STRUCTURED_POINTS with one more point than cells per axis, one cell-data
# array per field, x fastest, big-endian).
# ---------------------------------------------------------------------------
_VTK_TYPES = {np.dtype(np.float32): "float", np.dtype(np.float64): "double", np.dtype(np.int32): "int",
              np.dtype(np.int64): "vtktypeint64", np.dtype(np.uint8): "unsigned_char"}


def _host(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def write_vtk_cells(filename, cell_dims, arrays, title="fields"):
    """Legacy binary VTK of a uniform grid of ``cell_dims`` cells (2 or 3 ints)
    with one cell-data array per ``arrays`` entry (name -> array of that shape,
    or already flat in x-fastest order)."""
    dims = tuple(int(d) for d in cell_dims) + (1,) * (3 - len(cell_dims))
    ncell = int(np.prod(dims))
    with open(filename, "wb") as fh:
        fh.write(f"# vtk DataFile Version 3.0\n{title}\nBINARY\nDATASET STRUCTURED_POINTS\n".encode())
        fh.write("DIMENSIONS {} {} {}\n".format(*[d + 1 if d > 1 or i < len(cell_dims) else 1
                                                  for i, d in enumerate(dims)]).encode())
        fh.write(b"ORIGIN 0 0 0\nSPACING 1 1 1\n")
        fh.write(f"CELL_DATA {ncell}\n".encode())
        for name, a in arrays.items():
            a = _host(a)
            if a.dtype == np.bool_:
                a = a.astype(np.uint8)
            if a.dtype not in _VTK_TYPES:
                a = a.astype(np.float64)
            flat = a.reshape(-1, order="F") if a.ndim > 1 else a.reshape(-1)
            if flat.size != ncell:
                raise ValueError(f"field {name!r} has {flat.size} values for {ncell} cells")
            fh.write(f"SCALARS {name} {_VTK_TYPES[flat.dtype]} 1\nLOOKUP_TABLE default\n".encode())
            fh.write(flat.astype(flat.dtype.newbyteorder(">")).tobytes())
            fh.write(b"\n")


def save_fields_vtk(timestep, fields, output_dir=".", prefix="fields"):
    """``src/utils.py:144-196``: every field of ``fields`` (all the same shape,
    (nx, ny) or (nx, ny, nz)) as cell data of ``<prefix>_<timestep:07d>.vtk``."""
    shapes = {tuple(np.shape(_host(v))) for v in fields.values()}
    assert len(shapes) == 1, "All fields must have the same dimensions!"
    (shape,) = shapes
    output_filename = os.path.join(output_dir, prefix + "_" + f"{timestep:07d}.vtk")
    start = time.time()
    write_vtk_cells(output_filename, shape, fields, title=prefix)
    print(f"Saved {output_filename} in {time.time() - start:.6f} seconds.")


def save_BCs_vtk(timestep, BCs, gridInfo, output_dir="."):
    """``src/utils.py:243-304``: one boolean cell array per boundary condition
    (named ``<bc.name>_<k>`` for the k-th BC of that name) in ``BCs_<timestep:07d>.vtk``."""
    dims = (gridInfo["nx"], gridInfo["ny"]) if gridInfo["nz"] == 0 else \
        (gridInfo["nx"], gridInfo["ny"], gridInfo["nz"])
    counts, arrays = {}, {}
    for bc in BCs:
        counts[bc.name] = counts.get(bc.name, -1) + 1
        idx = bc.update_function(timestep)[0] if getattr(bc, "isDynamic", False) else bc.indices
        mask = np.zeros(dims, dtype=bool)
        mask[tuple(np.asarray(i) for i in idx)] = True
        arrays[f"{bc.name}_{counts[bc.name]}"] = mask
    output_filename = os.path.join(output_dir, "BCs_" + f"{timestep:07d}.vtk")
    start = time.time()
    write_vtk_cells(output_filename, dims, arrays, title="BCs")
    print(f"Saved {output_filename} in {time.time() - start:.6f} seconds.")
