"""D2Q8 / D2Q9 lattice constants (oracle).  Restates ``src/lattice.py``."""
import re
import numpy as np


def dtypes_for(precision):
    """Compute/storage dtypes of a precision string (``src/elasticity.py:606-629``,
    ``src/base.py`` set_precisions).  Unknown strings fall back to f32/f32."""
    return {
        "f64/f64": (np.float64, np.float64),
        "f32/f32": (np.float32, np.float32),
        "f32/f16": (np.float32, np.float16),
        "f16/f16": (np.float16, np.float16),
        "f64/f32": (np.float64, np.float32),
        "f64/f16": (np.float64, np.float16),
    }.get(precision, (np.float32, np.float32))


class Policy:
    """The jmp policy subset used by the reference (cast inputs to compute,
    outputs to storage; ``src/elasticity.py:63-66``)."""

    def __init__(self, precision):
        self.compute_dtype, self.output_dtype = dtypes_for(precision)
        self.param_dtype = self.compute_dtype

    def cast_to_compute(self, x):
        if isinstance(x, tuple):
            return tuple(self.cast_to_compute(v) for v in x)
        return None if x is None else np.asarray(x).astype(self.compute_dtype)

    def cast_to_output(self, x):
        return None if x is None else np.asarray(x).astype(self.output_dtype)


class Lattice:
    """``src/lattice.py:6-213``."""

    def __init__(self, name, precision="f32/f32"):
        self.name = name
        dq = re.findall(r"\d+", name)
        self.precision = precision
        self.d, self.q = int(dq[0]), int(dq[1])
        if precision in ("f32/f32", "f32/f16"):
            self.precisionPolicy = np.float32
        elif precision in ("f64/f64", "f64/f32", "f64/f16"):
            self.precisionPolicy = np.float64
        elif precision == "f16/f16":
            self.precisionPolicy = np.float16
        else:
            raise ValueError("precision not supported")
        if name == "D2Q8":      # src/lattice.py:124-127
            cx = [1, 0, -1, 0, 1, -1, -1, 1]
            cy = [0, 1, 0, -1, 1, 1, -1, -1]
        elif name == "D2Q9":    # src/lattice.py:128-131
            cx = [0, 0, 0, 1, -1, 1, -1, 1, -1]
            cy = [0, 1, -1, 0, 1, -1, 0, 1, -1]
        elif name not in ("D3Q19", "D3Q27"):
            raise ValueError("oracle supports D2Q8, D2Q9, D3Q19 and D3Q27")
        if self.d == 2:
            self.c = np.array([cx, cy], dtype=np.int8)
        else:                   # src/lattice.py:132-138: loop order x, y, z over (0, -1, 1)
            vel = [(x, y, z) for x in (0, -1, 1) for y in (0, -1, 1) for z in (0, -1, 1)]
            if name == "D3Q19":
                vel = [v for v in vel if np.linalg.norm(v) < 1.5]
            self.c = np.array(vel, dtype=np.int8).T
        cT = self.c.T.astype(np.int64)
        norm = np.linalg.norm(cT, axis=1)
        w = np.full(self.q, 1.0 / 36.0)                 # src/lattice.py:144-182
        if self.d == 2:
            w[norm < 1.1] = 1.0 / 9.0
            if name == "D2Q9":
                w[0] = 4.0 / 9.0
        elif name == "D3Q19":
            w[norm < 1.1] = 2.0 / 36.0
            w[0] = 1.0 / 3.0
        else:
            w[np.isclose(norm, 1.0, atol=1e-8)] = 2.0 / 27.0
            w[(norm > 1) & (norm <= np.sqrt(2))] = 1.0 / 54.0
            w[(norm > np.sqrt(2)) & (norm <= np.sqrt(3))] = 1.0 / 216.0
            w[0] = 8.0 / 27.0
        self.w = w.astype(self.precisionPolicy)
        self.opp_indices = np.array(                     # src/lattice.py:51-65
            [cT.tolist().index((-cT[i]).tolist()) for i in range(self.q)], dtype=np.int64)
        self.main_indices = np.nonzero(np.abs(cT).sum(axis=1) == 1)[0]
        self.right_indices = np.nonzero(cT[:, 0] == 1)[0]
        self.left_indices = np.nonzero(cT[:, 0] == -1)[0]

    def __str__(self):
        return self.name


class LatticeD2Q8(Lattice):
    """``src/lattice.py:215-234``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D2Q8", precision)


class LatticeD2Q9(Lattice):
    """``src/lattice.py:236-258``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D2Q9", precision)


class LatticeD3Q19(Lattice):
    """``src/lattice.py:261-285``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D3Q19", precision)


class LatticeD3Q27(Lattice):
    """``src/lattice.py:287-307``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D3Q27", precision)
