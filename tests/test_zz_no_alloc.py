"""The allocation-free Darcy sweep entry point against the regular one.

``xlbb_darcy_sweep_residual_noalloc`` serves callers that cannot allocate
device memory (a CUDA-graph capture in progress, a host runtime that lends the
library only its own input/output buffers, a fixed memory budget): its FP64
residual partials live in scratch built into the library.  Through the C ABI it
must give the same populations and residual as ``xlbb_darcy_sweep`` with
caller-provided partials followed by ``xlbb_reduce_sum``, on two calls in a row
(the second call finds the first call's leftovers in the shared scratch), and
both residuals must equal the FP64 sum of (f_out - f_in)^2 taken on the host.
Covered: FP64 and FP32, the collide-and-push launch and the row-marching launch
that a sweep takes when its post-streaming rules have no push words, and the
rejection of a launch with more CTAs than the scratch holds.
This file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

PUSH_SHAPE = (128, 1, 1, 8, 3)      # the default collide-and-push launch shape


@pytest.fixture
def push_shape():
    from xlb_biot_b200 import autotune
    saved = autotune.get_config(autotune.DARCY)
    autotune.set_config(autotune.DARCY, *PUSH_SHAPE)
    yield
    autotune.set_config(autotune.DARCY, **saved)


def _setup(precision, n=200):
    import xlb_biot_b200.api as G
    from xlb_biot_b200 import _lib
    from xlb_biot_b200.workloads import darcy_lognormal
    solver, _ = darcy_lognormal(G, n=n, ell=8.0, precision=precision)
    return solver, _lib


def _negating_rules(solver):
    """Post-streaming rules without push words: on one interior column every
    streamed population is negated (a "keep" rule that transforms the streamed
    value), so the sweep runs on the row-marching launch."""
    from xlb_biot_b200.bc_compile import CompiledRules
    L = solver._layout
    nx, ny, q = solver.nx, solver.ny, 9
    cells = np.stack([np.full(ny, nx // 2), np.arange(ny)], axis=1).astype(np.int64)
    code = np.full((ny, q), 2 * q + 2, dtype=np.uint8)       # NEG_KEEP in every direction
    cst = np.zeros((ny, q))
    rules = CompiledRules(q, ny, cells, code, cst, L.dtype, L.device, nx, push=True)
    assert rules.push is None
    return rules


def _sweep_struct(solver, _lib, f_in, f_out, ps):
    return _lib.DarcySweep(f_in.data_ptr(), f_out.data_ptr(), float(solver.omega), solver.omega_field.data_ptr(),
                           None, None, solver._pc.struct(), ps.struct(), None)


@pytest.mark.parametrize("precision", ["f64/f64", "f32/f32"])
@pytest.mark.parametrize("rules", ["push", "row_marching"])
def test_noalloc_matches_regular_entry_point_twice(push_shape, precision, rules):
    solver, _lib = _setup(precision)
    lib = _lib.lib()
    L = solver._layout
    grid = L.grid()
    dcode = _lib.dtype_code(L.dtype)
    stream = _lib.stream_ptr()
    ps = solver._ps if rules == "push" else _negating_rules(solver)
    probe = _sweep_struct(solver, _lib, L.empty(9), L.empty(9), ps)
    assert lib.xlbb_darcy_sweep_pipeline(dcode, grid, probe) == (3 if rules == "push" else 0)
    n = lib.xlbb_darcy_sweep_partials(dcode, grid, probe)
    assert 0 < n <= lib.xlbb_darcy_sweep_ctas(dcode, grid) and n <= 16384
    partials = torch.empty(lib.xlbb_darcy_sweep_ctas(dcode, grid), dtype=torch.float64, device="cuda")
    f = solver.assign_fields_sharded()
    ref_in, new_in = f, f
    for call in range(2):
        ref_out, new_out = L.empty(9), L.empty(9)
        ref_sum = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        new_sum = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        s = _sweep_struct(solver, _lib, ref_in, ref_out, ps)
        s.sumsq = partials.data_ptr()
        _lib.check(lib.xlbb_darcy_sweep(dcode, grid, s, stream), "xlbb_darcy_sweep")
        _lib.check(lib.xlbb_reduce_sum(partials.data_ptr(), n, ref_sum.data_ptr(), stream), "xlbb_reduce_sum")
        s2 = _sweep_struct(solver, _lib, new_in, new_out, ps)
        _lib.check(lib.xlbb_darcy_sweep_residual_noalloc(dcode, grid, s2, ctypes.c_void_p(new_sum.data_ptr()),
                                                         stream), "xlbb_darcy_sweep_residual_noalloc")
        torch.cuda.synchronize()
        a, b = ref_out.cpu().numpy(), new_out.cpu().numpy()
        assert np.array_equal(a, b), f"call {call}: populations differ"
        host = float(np.sum((a.astype(np.float64) - ref_in.cpu().numpy().astype(np.float64)) ** 2))
        r, q = float(ref_sum[0]), float(new_sum[0])
        assert host > 0 and abs(r - host) <= 1e-12 * host, f"call {call}: regular residual {r} != host sum {host}"
        assert abs(q - host) <= 1e-12 * host, f"call {call}: allocation-free residual {q} != host sum {host}"
        ref_in, new_in = ref_out, new_out


def test_noalloc_rejects_a_launch_larger_than_its_scratch(push_shape):
    """2048 x 2048 under the collide-and-push shape has 16 * 2048 CTAs."""
    solver, _lib = _setup("f32/f32", n=2048)
    lib = _lib.lib()
    L = solver._layout
    grid = L.grid()
    f_in, f_out = solver.assign_fields_sharded(), L.empty(9)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    s = _sweep_struct(solver, _lib, f_in, f_out, solver._ps)
    assert lib.xlbb_darcy_sweep_partials(_lib.XLBB_F32, grid, s) == 16 * 2048
    st = lib.xlbb_darcy_sweep_residual_noalloc(_lib.XLBB_F32, grid, s, ctypes.c_void_p(out.data_ptr()),
                                               _lib.stream_ptr())
    assert st == _lib.XLBB_EBADARG
    assert b"16384" in lib.xlbb_last_error()
    torch.cuda.synchronize()
    assert float(out[0]) == 0.0


def test_noalloc_rejects_bad_arguments():
    solver, _lib = _setup("f64/f64")
    s = _lib.DarcySweep()
    st = _lib.lib().xlbb_darcy_sweep_residual_noalloc(_lib.XLBB_F64, solver._layout.grid(), s, None, None)
    assert st == _lib.XLBB_EBADARG
