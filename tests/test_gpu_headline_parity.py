"""The benchmarked Darcy variant against the oracle, at the benchmark's sizes.

The headline workload (``workloads.darcy_lognormal``: log-normal permeability,
per-cell omega, pressure anti-bounce-back left/right, bounce-back top/bottom,
corner-patched masks) runs through the same CUDA-graph sweep loop as the bench
(collide-and-push launch, FP64 residual fused into the last sweep) and through
the oracle, from the same initial populations, on 256 x 256 and on the full
1024 x 1024 grid.  Relative difference of the populations (to max |f|):
<= 1e-12 in FP64, <= 1e-5 in FP32; the FP64 residual of the last sweep within
the same bounds of the oracle's sum((f_n - f_{n-1})^2).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SWEEPS = 20


@pytest.fixture
def push_shape():
    from xlb_biot_b200 import autotune
    saved = autotune.get_config(autotune.DARCY)
    autotune.set_config(autotune.DARCY, 128, 1, 1, 8, 3)
    yield
    autotune.set_config(autotune.DARCY, **saved)


@pytest.mark.parametrize("n", [256, 1024])
@pytest.mark.parametrize("prec,tol", [("f64/f64", 1e-12), ("f32/f32", 1e-5)])
def test_lognormal_darcy_matches_oracle(push_shape, n, prec, tol):
    import torch
    import oracle.api as O
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import darcy_lognormal
    so, _ = darcy_lognormal(O, n=n, precision=prec)
    sg, _ = darcy_lognormal(G, n=n, precision=prec)
    assert sg.omega_field is not None
    f0 = so.assign_fields_sharded()
    # a perturbed start so that every population and boundary rule carries signal
    f0 = (f0 + 1e-2 * np.random.default_rng(7).standard_normal(f0.shape)).astype(f0.dtype)

    fo = f0
    prev = None
    for t in range(SWEEPS):
        prev = fo
        fo, _ = so.step(fo, t)
    res_o = float(np.sum((fo.astype(np.float64) - prev.astype(np.float64)) ** 2))

    loop = sg.sweep_graph(SWEEPS)
    loop.state.copy_(sg._layout.field(f0, 9))
    assert sg.sweep_pipeline() == 3          # the collide-and-push launch of the bench
    out = loop.replay()
    torch.cuda.synchronize()
    fg = out.cpu().numpy()
    scale = np.abs(fo).max()
    err = np.abs(fg.astype(np.float64) - fo.astype(np.float64)).max() / scale
    assert err <= tol, f"{n}^2 {prec}: populations differ from the oracle by {err:.3e}"
    res_g = float(loop.sumsq[0])
    # FP32: the residual differences of O(1e-2) populations carry the FP32 rounding of each population
    rtol = 1e-10 if prec == "f64/f64" else 1e-3
    assert abs(res_g - res_o) <= rtol * res_o, f"{n}^2 {prec}: residual {res_g} vs oracle {res_o}"
