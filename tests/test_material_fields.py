"""Per-cell Lame fields (extension without a reference counterpart) on CPU.

* The oracle's per-cell material reduces to the reference restatement when
  the fields are uniform (every formula, every multigrid level).
* The product's coarse-level material (torch, differentiable) equals the
  oracle's ``coarsen_field`` for every MG_BCs combination.
"""
import numpy as np
import pytest
import torch

import oracle.api as O
from oracle.elasticity import coarsen_field
from xlb_biot_b200.workloads import terzaghi_heterogeneous


def _run(sim, steps):
    e, d, t = sim.init_state()
    out = None
    for k in range(steps):
        out = sim.step(e, d, t, k)
        e, d, t = out[0], out[1], out[4]
    return out


def test_uniform_fields_reduce_to_reference():
    z = np.zeros((16, 10))
    a, _ = terzaghi_heterogeneous(O, nx=16, ny=10, levels=3, cycles=2, precision="f64/f64", log_mu=z, log_k=z)
    b, _ = terzaghi_heterogeneous(O, nx=16, ny=10, levels=3, cycles=2, precision="f64/f64", log_mu=z, log_k=z)
    b.elasticity._fields = None                    # the reference's scalar path
    b.darcy.omega = float(np.asarray(b.darcy.omega).ravel()[0])
    oa, ob = _run(a, 3), _run(b, 3)
    for x, y in zip(oa, ob):
        x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
        assert np.abs(x - y).max() <= 1e-13 * max(np.abs(y).max(), 1e-300)


def test_heterogeneous_fields_change_the_solution():
    a, _ = terzaghi_heterogeneous(O, nx=16, ny=10, levels=3, cycles=2, precision="f64/f64", ell=3.0)
    z = np.zeros((16, 10))
    b, _ = terzaghi_heterogeneous(O, nx=16, ny=10, levels=3, cycles=2, precision="f64/f64", log_mu=z, log_k=z)
    oa, ob = _run(a, 3), _run(b, 3)
    assert np.all(np.isfinite(oa[0])) and np.abs(oa[0] - ob[0]).max() > 1e-3 * np.abs(ob[0]).max()


@pytest.mark.parametrize("bcs", [dict(bottom=True, top=True), dict(left=True, right=True),
                                 dict(left=True, right=True, bottom=True, top=True), {}])
def test_coarsen_material_matches_oracle(bcs):
    from xlb_biot_b200.elasticity import coarsen_material
    full = {"left": False, "right": False, "bottom": False, "top": False}
    full.update(bcs)
    nx = 16 + int(full["left"]) + int(full["right"])
    ny = 8 + int(full["bottom"]) + int(full["top"])
    a = np.random.default_rng(0).uniform(0.5, 2.0, (nx, ny))
    got = coarsen_material(torch.as_tensor(a), full).numpy()
    ref = coarsen_field(a, full)
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-15
