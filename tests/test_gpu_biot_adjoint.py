"""Adjoint of the heterogeneous consolidation time loop (FP64 and FP32).

* The adjoint driver's taped forward step equals ``LBMPoroelasticity.step``
  bit for bit.
* Gradients of the misfit with respect to log-shear-modulus and
  log-permeability fields (through ``ConsolidationMisfit`` and torch's
  autograd) agree with central finite differences along random directions.
* The checkpoint interval does not change the gradient.
* FP32 gradients agree with the FP64 ones.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
KW = dict(nx=32, ny=18, levels=3, cycles=2, k_smooth=2, ell=5.0, load=1e-2)
STEPS = 6


def _model(prec, every=4, seed=0, graphs=False):
    import xlb_biot_b200.api as G
    from xlb_biot_b200.biot_adjoint import BiotAdjointModel
    from xlb_biot_b200.workloads import terzaghi_heterogeneous
    sim, mat = terzaghi_heterogeneous(G, precision=prec, seed=seed, **KW)
    return BiotAdjointModel(sim, STEPS, checkpoint_every=every, graphs=graphs), mat


def _observations(prec):
    """The last step's displacement and pressure of a perturbed-material run."""
    model, mat = _model(prec, seed=5)
    model.forward()
    return model.eta.double().clone(), model.p.double().clone()


def _J_and_grad(model, mat, obs, dev, dtype=torch.float64):
    from xlb_biot_b200.biot_adjoint import ConsolidationMisfit, consolidation_parameters
    model.set_observations(*obs)
    lm = torch.as_tensor(mat["log_mu"], dtype=dtype, device=dev).requires_grad_()
    lk = torch.as_tensor(mat["log_k"], dtype=dtype, device=dev).requires_grad_()
    J = ConsolidationMisfit.apply(*consolidation_parameters(lm, lk), model)
    J.backward()
    return float(J.detach()), lm.grad.double(), lk.grad.double()


def _J(model, log_mu, log_k):
    from xlb_biot_b200.biot_adjoint import consolidation_parameters
    model.set_parameters(*consolidation_parameters(log_mu, log_k))
    return model.forward()


def test_taped_step_equals_solver_step():
    model, _ = _model("f64/f64")
    sim = model.sim
    a = sim.init_state()
    b = sim.init_state()
    for t in range(3):
        oa = sim.step(a[0], a[1], a[2], t)
        ob = model.step(b[0], b[1], b[2])
        a, b = (oa[0], oa[1], oa[4]), ob[:3]
    for x, y in zip(a, b):
        assert torch.equal(x.double(), y.double())
    assert torch.equal(oa[2].double(), ob[3].double()) and torch.equal(oa[5].double(), ob[4].double())


def test_gradient_matches_central_differences():
    dev = torch.device("cuda")
    obs = _observations("f64/f64")
    model, mat = _model("f64/f64")
    J, g_mu, g_k = _J_and_grad(model, mat, obs, dev)
    assert J > 0 and torch.isfinite(g_mu).all() and torch.isfinite(g_k).all()
    rng = np.random.default_rng(1)
    lm0 = torch.as_tensor(mat["log_mu"], dtype=torch.float64, device=dev)
    lk0 = torch.as_tensor(mat["log_k"], dtype=torch.float64, device=dev)
    for trial in range(3):
        dm = torch.as_tensor(rng.standard_normal(lm0.shape), device=dev)
        dk = torch.as_tensor(rng.standard_normal(lk0.shape), device=dev)
        eps = 1e-5
        jp = _J(model, lm0 + eps * dm, lk0 + eps * dk)
        jm = _J(model, lm0 - eps * dm, lk0 - eps * dk)
        fd = (jp - jm) / (2 * eps)
        ad = float((g_mu * dm).sum() + (g_k * dk).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd), (trial, fd, ad)


def test_checkpoint_interval_does_not_change_the_gradient():
    dev = torch.device("cuda")
    obs = _observations("f64/f64")
    res = []
    for every in (1, 4, 100):
        model, mat = _model("f64/f64", every=every)
        res.append(_J_and_grad(model, mat, obs, dev))
    for J, gm, gk in res[1:]:
        assert J == res[0][0]
        assert torch.allclose(gm, res[0][1], rtol=1e-12, atol=1e-12 * float(res[0][1].abs().max()))
        assert torch.allclose(gk, res[0][2], rtol=1e-12, atol=1e-12 * float(res[0][2].abs().max()))


def test_fp32_gradient_agrees_with_fp64():
    dev = torch.device("cuda")
    obs = _observations("f64/f64")
    m64, mat = _model("f64/f64")
    _, gm64, gk64 = _J_and_grad(m64, mat, obs, dev)
    m32, _ = _model("f32/f32")
    _, gm32, gk32 = _J_and_grad(m32, mat, obs, dev)
    for a, b in ((gm32, gm64), (gk32, gk64)):
        rel = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        assert rel < 1e-3, rel


@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_graph_mode_equals_eager(prec):
    """The CUDA-graph time loop (plain step, per-slot taping step and adjoint)
    replays exactly the eager kernels: J and gradients bit-identical, twice."""
    dev = torch.device("cuda")
    obs = _observations("f64/f64")
    me, mat = _model(prec, every=4)
    ref = _J_and_grad(me, mat, obs, dev)
    mg, _ = _model(prec, every=4, graphs=True)
    for _ in range(2):
        got = _J_and_grad(mg, mat, obs, dev)
        assert got[0] == ref[0]
        assert torch.equal(got[1], ref[1]) and torch.equal(got[2], ref[2])
