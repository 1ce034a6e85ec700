"""D2Q8 / D2Q9 lattices (mirror of ``src/lattice.py``; host-side constants).

The velocity sets, weights and index tables are the reference's
(``src/lattice.py:124-131,144-182,51-91``); they are kept as NumPy arrays
because they are consumed by the host-side boundary preprocessing, while the
kernels carry the same tables as compile-time constants.
"""
import re

import numpy as np


class Lattice:
    """``src/lattice.py:6-213`` for the 2D lattices of the Biot path."""

    _VEL = {"D2Q8": ([1, 0, -1, 0, 1, -1, -1, 1], [0, 1, 0, -1, 1, 1, -1, -1]),
            "D2Q9": ([0, 0, 0, 1, -1, 1, -1, 1, -1], [0, 1, -1, 0, 1, -1, 0, 1, -1])}

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
        if name not in self._VEL:
            raise ValueError("Supported lattice types on the Biot path are D2Q8 and D2Q9")
        self.c = np.array(self._VEL[name], dtype=np.int8)
        cT = self.c.T.astype(np.int64)
        norm = np.linalg.norm(cT, axis=1)
        w = np.where(norm < 1.1, 1.0 / 9.0, 1.0 / 36.0)
        if name == "D2Q9":
            w[0] = 4.0 / 9.0
        self.w = w.astype(self.precisionPolicy)
        self.cc = np.stack([cT[:, 0] * cT[:, 0], cT[:, 0] * cT[:, 1], cT[:, 1] * cT[:, 1]], axis=1).astype(
            self.precisionPolicy)
        self.opp_indices = np.array([int(np.nonzero((cT == -cT[i]).all(axis=1))[0][0]) for i in range(self.q)],
                                    dtype=np.int8)
        self.main_indices = np.nonzero(np.abs(cT[:, 0]) + np.abs(cT[:, 1]) == 1)[0].astype(np.int8)
        self.right_indices = np.nonzero(cT[:, 0] == 1)[0].astype(np.int8)
        self.left_indices = np.nonzero(cT[:, 0] == -1)[0].astype(np.int8)

    def __str__(self):
        return self.name


class LatticeD2Q8(Lattice):
    """``src/lattice.py:215-234``: D2Q8 without rest velocity (elasticity)."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D2Q8", precision)
        self.i_s = np.arange(8, dtype=np.int8)
        self.im = 2
        self.ik = 3


class LatticeD2Q9(Lattice):
    """``src/lattice.py:236-258``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D2Q9", precision)
        self.cs = np.sqrt(3) / 3.0
        self.cs2 = 1.0 / 3.0
        self.inv_cs2 = 3.0
        self.i_s = np.arange(9, dtype=np.int8)
        self.im = 3
        self.ik = 3
