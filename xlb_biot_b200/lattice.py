"""D2Q8 / D2Q9 / D3Q19 / D3Q27 lattices (mirror of ``src/lattice.py``; host-side constants).

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

    @staticmethod
    def _velocities(name):
        """``src/lattice.py:111-140``: the 2D tables, and for 3D every (x, y, z)
        in {0, -1, 1}^3 in that loop order (D3Q19: without the 8 corners)."""
        if name in Lattice._VEL:
            return np.array(Lattice._VEL[name], dtype=np.int8)
        if name in ("D3Q19", "D3Q27"):
            c = [(x, y, z) for x in (0, -1, 1) for y in (0, -1, 1) for z in (0, -1, 1)]
            if name == "D3Q19":
                c = [v for v in c if np.linalg.norm(v) < 1.5]
            return np.array(c, dtype=np.int8).T
        raise ValueError("Supported lattice types are D2Q8, D2Q9, D3Q19 and D3Q27")

    @staticmethod
    def _weights(name, cT):
        """``src/lattice.py:142-182``."""
        norm = np.linalg.norm(cT, axis=1)
        w = np.full(len(cT), 1.0 / 36.0)
        if name in ("D2Q8", "D2Q9"):
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
        return w

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
        self.c = self._velocities(name)
        cT = self.c.T.astype(np.int64)
        self.w = self._weights(name, cT).astype(self.precisionPolicy)
        # src/lattice.py:184-211: the independent products c_a c_b (a <= b)
        self.cc = np.stack([cT[:, a] * cT[:, b] for a in range(self.d) for b in range(a, self.d)],
                           axis=1).astype(self.precisionPolicy)
        self.opp_indices = np.array([int(np.nonzero((cT == -cT[i]).all(axis=1))[0][0]) for i in range(self.q)],
                                    dtype=np.int8)
        self.main_indices = np.nonzero(np.abs(cT).sum(axis=1) == 1)[0].astype(np.int8)
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


class LatticeD3Q19(Lattice):
    """``src/lattice.py:261-285``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D3Q19", precision)
        self.cs = np.sqrt(3) / 3.0
        self.cs2 = 1.0 / 3.0
        self.inv_cs2 = 3.0
        self.i_s = np.arange(19, dtype=np.int8)
        self.im = 9
        self.ik = 5


class LatticeD3Q27(Lattice):
    """``src/lattice.py:287-307``."""

    def __init__(self, precision="f32/f32"):
        super().__init__("D3Q27", precision)
        self.cs = np.sqrt(3) / 3.0
        self.cs2 = 1.0 / 3.0
        self.inv_cs2 = 3.0
        self.i_s = np.arange(27, dtype=np.int8)
