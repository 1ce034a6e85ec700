"""The allocation-free Darcy sweep entry point against the regular one.

``xlbb_darcy_sweep_residual_noalloc`` serves callers that cannot allocate
device memory (a CUDA-graph capture in progress, a host runtime that lends the
library only its own input/output buffers, a fixed memory budget): its FP64
residual partials live in scratch built into the library.  Through the C ABI it
must give the same populations and residual as ``xlbb_darcy_sweep`` with
caller-provided partials followed by ``xlbb_reduce_sum``, on two calls in a row
(the second call finds the first call's leftovers in the shared scratch).
This file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup():
    import xlb_biot_b200.api as G
    from xlb_biot_b200 import _lib
    from xlb_biot_b200.workloads import darcy_lognormal
    solver, _ = darcy_lognormal(G, n=200, ell=8.0, precision="f64/f64")
    return solver, _lib


def _sweep_struct(solver, _lib, f_in, f_out):
    return _lib.DarcySweep(f_in.data_ptr(), f_out.data_ptr(), float(solver.omega), solver.omega_field.data_ptr(),
                           None, None, solver._pc.struct(), solver._ps.struct(), None)


def test_noalloc_matches_regular_entry_point_twice():
    solver, _lib = _setup()
    lib = _lib.lib()
    L = solver._layout
    grid = L.grid()
    stream = _lib.stream_ptr()
    n = lib.xlbb_darcy_sweep_ctas(_lib.XLBB_F64, grid)
    assert 0 < n <= 16384
    partials = torch.empty(n, dtype=torch.float64, device="cuda")
    f = solver.assign_fields_sharded()
    ref_in, new_in = f, f
    for call in range(2):
        ref_out, new_out = L.empty(9), L.empty(9)
        ref_sum = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        new_sum = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        s = _sweep_struct(solver, _lib, ref_in, ref_out)
        s.sumsq = partials.data_ptr()
        _lib.check(lib.xlbb_darcy_sweep(_lib.XLBB_F64, grid, s, stream), "xlbb_darcy_sweep")
        _lib.check(lib.xlbb_reduce_sum(partials.data_ptr(), n, ref_sum.data_ptr(), stream), "xlbb_reduce_sum")
        s2 = _sweep_struct(solver, _lib, new_in, new_out)
        _lib.check(lib.xlbb_darcy_sweep_residual_noalloc(_lib.XLBB_F64, grid, s2, ctypes.c_void_p(new_sum.data_ptr()),
                                                         stream), "xlbb_darcy_sweep_residual_noalloc")
        torch.cuda.synchronize()
        a, b = ref_out.cpu().numpy(), new_out.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), f"call {call}: populations differ"
        r, q = float(ref_sum[0]), float(new_sum[0])
        assert r > 0 and abs(r - q) <= 1e-12 * r, f"call {call}: residual {q} != {r}"
        ref_in, new_in = ref_out, new_out


def test_noalloc_rejects_bad_arguments():
    solver, _lib = _setup()
    s = _lib.DarcySweep()
    st = _lib.lib().xlbb_darcy_sweep_residual_noalloc(_lib.XLBB_F64, solver._layout.grid(), s, None, None)
    assert st == -1
