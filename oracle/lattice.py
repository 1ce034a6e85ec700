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
        else:
            raise ValueError("oracle supports D2Q8 and D2Q9")
        self.c = np.array([cx, cy], dtype=np.int8)
        cT = self.c.T.astype(np.int64)
        w = np.full(self.q, 1.0 / 36.0)                 # src/lattice.py:144-182
        w[np.linalg.norm(cT, axis=1) < 1.1] = 1.0 / 9.0
        if name == "D2Q9":
            w[0] = 4.0 / 9.0
        self.w = w.astype(self.precisionPolicy)
        self.opp_indices = np.array(                     # src/lattice.py:51-65
            [cT.tolist().index((-cT[i]).tolist()) for i in range(self.q)], dtype=np.int64)
        self.main_indices = np.nonzero(np.abs(cT[:, 0]) + np.abs(cT[:, 1]) == 1)[0]
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
