"""Failure detection on the GPU, in the forms that fault and hang nothing.

* Bounded waits: ``xlbb_wait_selftest`` waits on an mbarrier that nothing
  completes with a limit of a few polls; the wait gives up, the kernel returns,
  ``xlbb_device_status`` reports XLBB_ETIMEOUT and the context stays usable.
* Non-finite fields: a NaN planted in the populations (or an instance's force)
  makes every tolerance solve raise ``NonFiniteError`` at its first check
  instead of iterating to its limit, and the FP64 reduction records
  XLBB_ENONFINITE in the device status word.
"""
import sys
import os

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.dirname(__file__))
from problems import elastic_material, make_darcy, make_periodic_elasticity  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def clean_status():
    from xlb_biot_b200 import autotune
    autotune.device_status(reset=True)
    yield
    autotune.device_status(reset=True)


def test_bounded_wait_gives_up_and_the_context_stays_usable():
    import xlb_biot_b200.api as G
    from xlb_biot_b200 import _lib, autotune
    lib = _lib.lib()
    gave_up = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lib.xlbb_wait_selftest(64, gave_up.data_ptr(), _lib.stream_ptr()), "xlbb_wait_selftest")
    torch.cuda.synchronize()
    assert int(gave_up[0]) == 1
    assert autotune.device_status(reset=True) == _lib.XLBB_ETIMEOUT
    assert autotune.device_status(reset=False) == 0
    assert lib.xlbb_wait_selftest(0, gave_up.data_ptr(), _lib.stream_ptr()) == _lib.XLBB_EBADARG
    # the context still runs kernels
    D = make_darcy(G, "anti")(lattice=G.LatticeD2Q9("f64/f64"), omega=1.25, nx=20, ny=20, nz=0,
                              precision="f64/f64")
    f, _ = D.step(D.assign_fields_sharded(), 1)
    torch.cuda.synchronize()
    assert torch.isfinite(f).all()
    assert autotune.device_status(reset=False) == 0


def _expect_nonfinite(run):
    from xlb_biot_b200 import _lib, autotune
    with pytest.raises(_lib.NonFiniteError):
        run()
    torch.cuda.synchronize()
    assert autotune.device_status(reset=True) == _lib.XLBB_ENONFINITE


@pytest.mark.parametrize("prec", ["f64/f64", "f32/f32"])
def test_darcy_solve_stops_on_nan(prec):
    import xlb_biot_b200.api as G
    D = make_darcy(G, "anti")(lattice=G.LatticeD2Q9(prec), omega=1.25, nx=24, ny=20, nz=0, precision=prec)
    f0 = D.assign_fields_sharded().clone()
    f0[5, 7, 3] = float("nan")
    _expect_nonfinite(lambda: D.solve(f0, tol=1e-12, check_every=10, max_sweeps=10 ** 7))


@pytest.mark.parametrize("levels", [1, 2])
def test_elasticity_solve_stops_on_nan(levels):
    import xlb_biot_b200.api as G
    lam, mu = elastic_material()
    E = make_periodic_elasticity(G)(lattice=G.LatticeD2Q8("f64/f64"), **{"lambda": lam}, mu=mu, nx=16, ny=16, nz=0,
                                    precision="f64/f64", MG_levels=levels)
    f0 = E.assign_fields_sharded().clone()
    f0[2, 3, 1] = float("nan")
    _expect_nonfinite(lambda: E.solve(f0, tol=1e-12, check_every=10, max_sweeps=10 ** 7))


def test_batched_solve_names_the_instance_with_nan():
    from xlb_biot_b200 import _lib
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=4, sizes=(32, 48), seed=2)
    forces = [np.array(f, copy=True) for f in forces]
    forces[2][4, 4, 0] = np.nan
    b = BatchedElasticity(sizes, lams, mus, forces, levels=3, precision="f32/f32")
    with pytest.raises(_lib.NonFiniteError, match=r"instances \[2\]"):
        b.solve(tol=1e-10, max_cycles=10 ** 6)
