"""Failure detection on the host: the loop driver of every tolerance solve
(``solve`` of the elasticity, Darcy and batched solvers) stops at the first
non-finite residual with ``NonFiniteError`` (XLBB_ENONFINITE) instead of
iterating to its limit, reports the rounding-floor stall, and the C-ABI status
mapping raises the same error class.  No GPU: the device side is replaced by
plain callables that inject NaN / Inf into the residual sequence."""
import numpy as np
import pytest

from xlb_biot_b200 import _lib
from xlb_biot_b200._common import iterate_to_tolerance, require_finite


def _sequence(values, per_call=10):
    calls = {"n": 0}

    def advance():
        v = values[calls["n"]]
        calls["n"] += 1
        return per_call, v
    return advance, calls


def test_converging_sequence_stops_below_tolerance():
    advance, calls = _sequence([1e-2, 1e-4, 1e-6, 1e-9, 1e-12])
    it, rel, stalled = iterate_to_tolerance(advance, 1e-8, 10 ** 6)
    assert (it, rel, stalled) == (40, 1e-9, False) and calls["n"] == 4


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_residual_raises_at_once(bad):
    advance, calls = _sequence([1e-2, 1e-3, bad, 1e-5, 1e-6])
    with pytest.raises(_lib.NonFiniteError) as e:
        iterate_to_tolerance(advance, 1e-8, 10 ** 7)
    assert calls["n"] == 3                       # no iteration after the bad residual
    assert e.value.code == _lib.XLBB_ENONFINITE
    assert "after 30 iterations" in str(e.value)


def test_nan_never_loops_to_the_limit():
    """A NaN compares False with every tolerance: without the check the loop
    would run to max_iters."""
    advance, calls = _sequence([np.nan] * 1000, per_call=1)
    with pytest.raises(_lib.NonFiniteError):
        iterate_to_tolerance(advance, 1e-8, 10 ** 7, stall_checks=20)
    assert calls["n"] == 1


def test_stall_at_rounding_floor():
    vals = [1e-2, 1e-3, 1e-4, 1.3e-5] + [1.31e-5, 1.29e-5] * 20
    advance, calls = _sequence(vals)
    it, rel, stalled = iterate_to_tolerance(advance, 1e-8, 10 ** 6, stall_checks=5)
    assert stalled and rel > 1e-8 and calls["n"] == 9


def test_iteration_limit():
    advance, calls = _sequence([0.5] * 100, per_call=7)
    it, rel, stalled = iterate_to_tolerance(advance, 1e-8, 50)
    assert it == 56 and not stalled and calls["n"] == 8


def test_per_instance_measure_names_the_bad_instances():
    rel = np.array([1e-3, np.nan, 2e-3, np.inf, 1e-4])
    with pytest.raises(_lib.NonFiniteError, match=r"instances \[1, 3\]"):
        require_finite(rel, "relative V-cycle residual", 7)
    require_finite(np.array([1.0, 0.0]), "x", 1)          # finite values pass


def test_host_field_with_nan_is_caught_by_its_residual():
    """A NaN planted in a host-built field: the FP64 norm of any field that
    contains it is NaN, and the check raises."""
    f = np.random.default_rng(0).standard_normal((16, 16, 9))
    f[3, 5, 2] = np.nan
    with pytest.raises(_lib.NonFiniteError):
        require_finite(np.sqrt(np.sum(f.astype(np.float64) ** 2)), "residual norm", 1)


def test_abi_status_maps_to_error_class():
    with pytest.raises(_lib.NonFiniteError):
        _lib.check(_lib.XLBB_ENONFINITE, "xlbb_reduce_sum")
    with pytest.raises(_lib.XlbbError) as e:
        _lib.check(_lib.XLBB_ETIMEOUT, "xlbb_darcy_sweep")
    assert not isinstance(e.value, _lib.NonFiniteError) and e.value.code == _lib.XLBB_ETIMEOUT
