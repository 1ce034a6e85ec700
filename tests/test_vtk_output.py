"""Legacy-VTK output (``save_fields_vtk``, ``save_BCs_vtk``) read back on CPU:
header, grid dimensions, cell counts and the arrays in x-fastest order."""
import numpy as np

from xlb_biot_b200.utils import save_BCs_vtk, save_fields_vtk


def _read(path):
    raw = open(path, "rb").read()
    out, pos, header = {}, 0, []

    def line():
        nonlocal pos
        end = raw.index(b"\n", pos)
        s = raw[pos:end].decode()
        pos = end + 1
        return s
    for _ in range(7):
        header.append(line())
    ncell = int(line().split()[1])
    types = {"float": ">f4", "double": ">f8", "unsigned_char": ">u1", "int": ">i4"}
    while pos < len(raw):
        _, name, typ, _ = line().split()
        line()                                  # LOOKUP_TABLE default
        dt = np.dtype(types[typ])
        out[name] = np.frombuffer(raw[pos:pos + ncell * dt.itemsize], dtype=dt)
        pos += ncell * dt.itemsize + 1
    return header, ncell, out


def test_fields_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    eta_x, p = rng.standard_normal((5, 3)), rng.standard_normal((5, 3)).astype(np.float32)
    save_fields_vtk(12, {"eta_x": eta_x, "p": p}, str(tmp_path))
    header, ncell, arrays = _read(tmp_path / "fields_0000012.vtk")
    assert header[0].startswith("# vtk DataFile") and header[2] == "BINARY"
    assert header[3] == "DATASET STRUCTURED_POINTS" and header[4] == "DIMENSIONS 6 4 1"
    assert ncell == 15
    np.testing.assert_array_equal(arrays["eta_x"], eta_x.flatten(order="F"))
    np.testing.assert_array_equal(arrays["p"], p.flatten(order="F"))


def test_bcs_roundtrip(tmp_path):
    class BC:
        def __init__(self, name, idx):
            self.name, self.indices, self.isDynamic = name, idx, False
    bcs = [BC("BB", (np.array([0, 1]), np.array([0, 0]))), BC("BB", (np.array([3]), np.array([2]))),
           BC("Anti", (np.array([4]), np.array([1])))]
    save_BCs_vtk(3, bcs, {"nx": 5, "ny": 3, "nz": 0}, str(tmp_path))
    _, ncell, arrays = _read(tmp_path / "BCs_0000003.vtk")
    assert ncell == 15 and set(arrays) == {"BB_0", "BB_1", "Anti_0"}
    m = np.zeros((5, 3), bool)
    m[[0, 1], [0, 0]] = True
    np.testing.assert_array_equal(arrays["BB_0"].astype(bool), m.flatten(order="F"))
    assert arrays["Anti_0"].sum() == 1 and arrays["Anti_0"][4 + 5 * 1] == 1
