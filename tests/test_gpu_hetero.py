"""Heterogeneous Terzaghi-type consolidation (per-cell shear modulus and
permeability, the adjoint workload's forward model) against the oracle's
FP64 extension: all seven outputs of the coupled step after several steps,
and the graph-captured step bit-identical to the eager one."""
import numpy as np
import pytest
import torch

import oracle.api as O
from xlb_biot_b200.workloads import terzaghi_heterogeneous

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = (a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, np.float64))
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("prec,tol", [("f64/f64", 1e-11), ("f32/f32", 2e-5)])
def test_heterogeneous_consolidation_matches_oracle(prec, tol):
    import xlb_biot_b200.api as G
    kw = dict(nx=32, ny=18, levels=3, cycles=2, ell=5.0, load=1e-2)
    so, _ = terzaghi_heterogeneous(O, precision="f64/f64", **kw)
    sg, _ = terzaghi_heterogeneous(G, precision=prec, **kw)
    eo, do, to = so.init_state()
    eg, dg, tg = sg.init_state()
    for t in range(4):
        oo = so.step(eo, do, to, t)
        og = sg.step(eg, dg, tg, t)
        eo, do, to = oo[0], oo[1], oo[4]
        eg, dg, tg = og[0], og[1], og[4]
    for k, (a, b) in enumerate(zip(og, oo)):
        assert _rel(a, b) < tol, (k, _rel(a, b))


def test_heterogeneous_step_graph_matches_eager():
    import xlb_biot_b200.api as G
    sim, _ = terzaghi_heterogeneous(G, nx=32, ny=18, levels=3, cycles=2, ell=5.0, precision="f64/f64")
    graph = sim.capture_step(*sim.init_state())
    graph.load(*sim.init_state())
    e, d, t = sim.init_state()
    for step in range(3):
        eager = sim.step(e, d, t, step)
        e, d, t = eager[0], eager[1], eager[4]
        got = graph.replay()
    for k, (a, b) in enumerate(zip(got, eager)):
        assert torch.equal(a.double(), b.double()), k
