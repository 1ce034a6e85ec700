"""The oracle against fixtures produced by the reference's own solver source.

``tests/golden/reference_fixtures.npz`` holds the outputs of the unmodified
reference modules (s-lunowa/xlb-biot ``src/*.py``) run on the golden cases of
``tests/golden/cases.py`` in FP64 (generated by ``tests/golden/make_golden.py``
with a NumPy stand-in for the JAX array API, since JAX itself is not
installable).  The oracle must reproduce every array to 1e-12 relative to its
maximum (1e-5 for the cases under the 'f64/f32' policy, FP32 storage):
plain and multigrid elasticity with every BC family, the four Darcy
set-ups with moments and gradient, per-cell relaxation, periodic and
Terzaghi Biot runs (every step's outputs), multigrid transfers and equilibrium.
"""
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, TOLERANCE  # noqa: E402

FIXTURES = os.path.join(HERE, "golden", "reference_fixtures.npz")


def load(name):
    data = np.load(FIXTURES)
    pre = name + "/"
    return {k[len(pre):]: data[k] for k in data.files if k.startswith(pre)}


def oracle_namespace():
    import oracle.api as O
    from xlb_biot_b200.utils import Parameters     # host-only class of the product (no oracle copy)
    m = SimpleNamespace(**{k: getattr(O, k) for k in dir(O) if not k.startswith("_")})
    m.golden_set_omega = lambda solver, om: setattr(solver, "omega", om)
    m.Parameters = Parameters
    return m


def compare(got, ref, name, tol):
    assert set(got) == set(ref), (name, sorted(got), sorted(ref))
    for k, r in ref.items():
        g = np.asarray(got[k], dtype=np.float64)
        assert g.shape == r.shape, (name, k, g.shape, r.shape)
        scale = np.abs(r).max()
        err = np.abs(g - r).max() / scale if scale > 0 else np.abs(g).max()
        assert err <= tol, f"{name}/{k}: {err:.3e} > {tol}"


def test_fixtures_cover_every_case():
    data = np.load(FIXTURES)
    names = {k.split("/")[0] for k in data.files}
    assert names == set(CASES)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_reference_fixture(name):
    compare(CASES[name](oracle_namespace()), load(name), name, TOLERANCE[name])
