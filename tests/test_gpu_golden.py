"""The CUDA path against fixtures produced by the reference's own solver source.

Every golden case (``tests/golden/cases.py``) runs through the drop-in classes
and the C ABI on the GPU in FP64 and must match the reference's outputs
(``tests/golden/reference_fixtures.npz``, made by ``tests/golden/make_golden.py``
from the unmodified reference modules) to 1e-12 relative to each array's
maximum (FP32-storage cases: 1e-5) -- the same bar as the oracle, without the
oracle in between.
"""
import os
import sys
from types import SimpleNamespace

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, TOLERANCE  # noqa: E402
from test_golden_reference import compare, load  # noqa: E402

pytestmark = pytest.mark.gpu


def product_namespace():
    import xlb_biot_b200.api as G
    m = SimpleNamespace(**{k: getattr(G, k) for k in dir(G) if not k.startswith("_")})
    m.golden_cell_omega = "field"
    return m


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_reproduces_reference_fixture(name):
    import torch
    got = CASES[name](product_namespace())
    torch.cuda.synchronize()
    compare(got, load(name), name, TOLERANCE[name])
