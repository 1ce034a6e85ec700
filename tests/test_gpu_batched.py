"""Batched multigrid against independent single-instance solvers.

Every instance of a heterogeneous batch (sizes, Lame parameters, forces) must
follow the single-instance ``LBMElasticity`` V-cycle (which is itself checked
against the oracle) after the same number of cycles, and its level-0 residual
norm must match.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def G_c8():
    from xlb_biot_b200.lattice import LatticeD2Q8
    return LatticeD2Q8("f64/f64").c


def _single(G, n, lam, mu, force, prec, levels, cycles, coarsest_precision=None, residual_precision=None):
    class E(G.LBMElasticity):
        def get_force(self):
            return self.distributed_array_init((n, n, 2), self.precisionPolicy.compute_dtype, init_val=force)
    s = E(lattice=G.LatticeD2Q8(prec), **{"lambda": float(lam)}, mu=float(mu), nx=n, ny=n, nz=0, precision=prec,
          MG_levels=levels, coarsest_precision=coarsest_precision, residual_precision=residual_precision,
          print_info_rate=0)
    f = s.assign_fields_sharded()
    norms = []
    for t in range(cycles):
        f, r = s.step(f, t)
        norms.append(float(r))
    return f.double().cpu().numpy(), norms


@pytest.mark.parametrize("prec,tol", [("f64/f64", 1e-12), ("f32/f32", 1e-5)])
def test_batched_vcycles_match_single_instances(prec, tol):
    import xlb_biot_b200.api as G
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=5, sizes=(32, 48, 64, 160), seed=3)
    b = BatchedElasticity(sizes, lams, mus, forces, levels=3, precision=prec)
    b.reset()
    norms = []
    for c in range(3):
        b.vcycle()
        norms.append(torch.sqrt(b.norm2).cpu().numpy().copy())
    for i, (nx, ny) in enumerate(sizes):
        f, ns = _single(G, nx, lams[i], mus[i], forces[i], prec, 3, 3)
        got = b.populations(i).double().cpu().numpy()
        assert np.abs(got - f).max() <= tol * np.abs(f).max(), i
        for c in range(3):
            assert abs(norms[c][i] - ns[c]) <= 10 * tol * ns[c], (i, c)


def test_batched_solve_converges():
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=8, sizes=(64, 96), seed=1)
    b = BatchedElasticity(sizes, lams, mus, forces, levels=4, precision="f32/f32", coarsest_precision="f64")
    cycles, rel = b.solve(tol=1e-4, max_cycles=80)
    assert np.all(rel < 1e-4) and cycles < 80


@pytest.mark.parametrize("prec,tol,rp", [("f64/f64", 1e-12, None), ("f32/f32", 1e-5, None), ("f32/f32", 1e-5, "f64")])
def test_batched_per_instance_levels_fp64_coarsest(prec, tol, rp):
    """Instances with different level counts (their coarsest levels at different
    depths, each in FP64) against single-instance solvers with the same levels
    (and, with rp="f64", FP64 arithmetic in both level-0 residual sweeps)."""
    import xlb_biot_b200.api as G
    from xlb_biot_b200.batched import BatchedElasticity, auto_levels
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=6, sizes=(24, 32, 48, 64), seed=5)
    b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision=prec, coarsest_precision="f64",
                          residual_precision=rp)
    assert b.instance_levels == [auto_levels(nx, ny) for nx, ny in sizes]
    assert len(set(b.instance_levels)) > 1
    b.reset()
    norms = []
    for c in range(3):
        b.vcycle()
        norms.append(torch.sqrt(b.norm2).cpu().numpy().copy())
    for i, (nx, ny) in enumerate(sizes):
        f, ns = _single(G, nx, lams[i], mus[i], forces[i], prec, b.instance_levels[i], 3, coarsest_precision="f64",
                        residual_precision=rp)
        got = b.populations(i).double().cpu().numpy()
        assert np.abs(got - f).max() <= tol * np.abs(f).max(), i
        for c in range(3):
            assert abs(norms[c][i] - ns[c]) <= 10 * tol * ns[c], (i, c)


def test_error_criterion_reaches_fp64_accuracy():
    """FP32 batch with the FP64-arithmetic level-0 residual, stopped by the
    estimated-error criterion at 1e-6 and ending with the removal of the
    drifted rigid-displacement mode: every instance's displacement is within
    1e-6 of an all-FP64 batch solved to 1e-11."""
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=12, sizes=(32, 48, 64, 96), seed=2)
    b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f32/f32", coarsest_precision="f64",
                          residual_precision="f64")
    cycles, est = b.solve(tol=1e-6, max_cycles=200, criterion="error")
    assert cycles < 200 and np.all(b.converged_at > 0)
    b64 = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f64/f64")
    c64, rel64 = b64.solve(tol=1e-11, max_cycles=400)
    assert np.all(rel64 < 1e-11)
    for i in range(len(sizes)):
        u, u64 = b.displacement(i), b64.displacement(i)
        err = float(torch.linalg.vector_norm(u - u64) / torch.linalg.vector_norm(u64))
        assert err < 1e-6, (i, err)


@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_remove_mean_moment_shifts_only_the_first_moments(prec):
    """``remove_mean_moment`` on random populations: afterwards every instance's
    mean first moments are zero, and each population moved by exactly
    (cx_i m_x + cy_i m_y) / 6 with m the mean before -- the other moments of
    every cell are unchanged."""
    from xlb_biot_b200.batched import BatchedElasticity
    sizes = [(16, 16), (24, 40), (64, 32)]
    forces = [np.zeros((nx, ny, 2)) for nx, ny in sizes]
    b = BatchedElasticity(sizes, [1.0] * 3, [1.0] * 3, forces, levels=2, precision=prec)
    g = torch.Generator(device="cuda").manual_seed(3)
    (arena,) = b.X[0].values()
    arena.buf.copy_(torch.rand(arena.buf.shape, generator=g, device="cuda", dtype=arena.buf.dtype) + 0.25)
    c = torch.as_tensor(np.asarray(G_c8(), dtype=np.float64), device="cuda")
    before = [b.populations(i).double().clone() for i in range(3)]
    b.remove_mean_moment()
    torch.cuda.synchronize()
    eps = 1e-13 if prec == "f64/f64" else 2e-7
    for i in range(3):
        f0, f1 = before[i], b.populations(i).double()
        m = torch.einsum("xyq,dq->d", f0, c) / (f0.shape[0] * f0.shape[1])
        expect = f0 - torch.einsum("d,dq->q", m, c) / 6.0
        assert float((f1 - expect).abs().max()) <= eps * float(f0.abs().max()), i
        assert float(torch.einsum("xyq,dq->d", f1, c).abs().max()) <= 10 * eps * float(f0.abs().sum()), i


@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_batched_push_and_row_marching_identical(prec):
    """The batched sweep's collide-and-push form (the default) and its
    row-marching form give bit-identical V-cycles (populations and correction
    norms); the residual norms group their FP64 partials differently."""
    from xlb_biot_b200 import autotune
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=5, sizes=(24, 32, 48, 64), seed=9)
    saved = autotune.get_config(autotune.ELASTICITY)
    out = []
    try:
        for shape in ((256, 1, 3, 8, 0), (128, 1, 1, 8, 3)):
            autotune.set_config(autotune.ELASTICITY, *shape)
            b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision=prec, coarsest_precision="f64",
                                  residual_precision="f64", vectorized=False)
            b.reset()
            for _ in range(3):
                b.vcycle()
            out.append(([b.populations(i).clone() for i in range(len(sizes))], b.norm2.clone(), b.corr2.clone()))
    finally:
        autotune.set_config(autotune.ELASTICITY, **saved)
    for x, y in zip(out[0][0], out[1][0]):
        assert torch.equal(x, y)
    assert torch.allclose(out[0][1], out[1][1], rtol=1e-12, atol=0) and torch.equal(out[0][2], out[1][2])


def _mixed_batch(seed=5):
    """Widths on one tile (64, 96, 24), on several (192, 256) and with a short
    last tile (136 = 128 + 8); coarse levels of 24 (6, 3) and of 136 (34, 17)
    are not multiples of 4 and stay on the one-column kernel."""
    rng = np.random.default_rng(seed)
    sizes = [(64, 40), (192, 64), (256, 32), (96, 48), (24, 24), (136, 72)]
    mus = rng.uniform(0.5, 2.0, len(sizes)) / 16.0
    nus = rng.uniform(0.1, 0.4, len(sizes))
    lams = 2 * mus * nus / (1 - nus)
    forces = [1e-3 * rng.standard_normal((nx, ny, 2)) for nx, ny in sizes]
    return sizes, lams, mus, forces


@pytest.mark.parametrize("rp", [None, "f64"])
def test_batched_four_column_kernel_identical(rp):
    """xlbb_batched_elast_sweep4 (four columns per lane, shuffles along x) and
    the one-column batched sweep give bit-identical V-cycles: populations and
    correction norms; the residual norms group their FP64 partials differently."""
    from xlb_biot_b200.batched import BatchedElasticity
    sizes, lams, mus, forces = _mixed_batch()
    out = []
    for vec in (False, True):
        b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f32/f32", coarsest_precision="f64",
                              residual_precision=rp, vectorized=vec)
        assert any(ln.vec for lns in b.smooth_xy for ln in lns) == vec
        b.reset()
        for _ in range(3):
            b.vcycle()
        out.append(([b.populations(i).clone() for i in range(len(sizes))], b.norm2.clone(), b.corr2.clone()))
    for i, (x, y) in enumerate(zip(out[0][0], out[1][0])):
        assert torch.equal(x, y), i
    assert torch.allclose(out[0][1], out[1][1], rtol=1e-12, atol=0) and torch.equal(out[0][2], out[1][2])


def test_four_column_kernel_skips_instances_that_do_not_qualify():
    """An instance whose width is not a multiple of 4, given to the four-column
    entry point, is skipped (its output untouched) and the device status word
    reports XLBB_EBADARG."""
    import ctypes
    from xlb_biot_b200 import _lib, autotune
    from xlb_biot_b200.batched import BatchedElasticity
    sizes = [(34, 34)]
    b = BatchedElasticity(sizes, [0.05], [0.05], [np.zeros((34, 34, 2))], levels=2, precision="f32/f32")
    ln = b.smooth_xy[0][0]
    assert not ln.vec
    dst = b.Y[0][torch.float32].view(0)
    dst.fill_(7.0)
    autotune.device_status(reset=True)
    lib = _lib.lib()
    _lib.check(lib.xlbb_batched_elast_sweep4(ln.dcode, ctypes.c_void_p(ln.desc.data_ptr()),
                                             ctypes.c_void_p(ln.tiles.data_ptr()), ln.ntiles, ln.ctas, 0.25, 0.75,
                                             1, 0, 0, None, 0, _lib.stream_ptr()), "xlbb_batched_elast_sweep4")
    torch.cuda.synchronize()
    assert autotune.device_status(reset=True) == -1        # XLBB_EBADARG
    assert bool((dst == 7.0).all())


@pytest.mark.parametrize("prec,coarse", [("f64/f64", None), ("f32/f32", None), ("f32/f32", "f64")])
@pytest.mark.parametrize("budget", [40 * 1024, 128 * 1024])
def test_persistent_tail_equals_level_by_level(prec, coarse, budget):
    """The coarse levels finished by one launch (a CTA per instance, levels in
    shared memory) give the level-by-level launches' populations and residual
    norms bit for bit, with fewer launches per V-cycle."""
    from xlb_biot_b200 import autotune
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=7, sizes=(32, 48, 64, 96, 128), seed=5)
    kw = dict(levels="auto", precision=prec, coarsest_precision=coarse)
    a = BatchedElasticity(sizes, lams, mus, forces, persistent_tail=True, tail_smem=budget, **kw)
    b = BatchedElasticity(sizes, lams, mus, forces, persistent_tail=False, **kw)
    assert a.tail is not None and b.tail is None
    assert all(1 <= t <= lv for t, lv in zip(a.tail_start, a.instance_levels))
    autotune.device_status(reset=True)
    a.reset()
    b.reset()
    for _ in range(3):
        a.vcycle()
        b.vcycle()
    torch.cuda.synchronize()
    assert autotune.device_status(reset=True) == 0
    assert a.launches_per_cycle < b.launches_per_cycle
    assert torch.equal(a.norm2, b.norm2)
    for i in range(len(sizes)):
        assert torch.equal(a.populations(i), b.populations(i)), i
