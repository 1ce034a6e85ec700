"""``.npz`` result caching of the convergence sweeps
(``examples/poroelasticity/periodic.py:217-259``): a run's error arrays are
saved under the example's file name and loaded instead of recomputed."""
import os

import numpy as np

from xlb_biot_b200.utils import cached_results, results_filename


def test_filename_follows_the_example():
    f = results_filename("/out", 0.11, 0.8, 0.1, 1.0, 32, 8, 5, "centered", alternative_gradient=True)
    assert f == os.path.join("/out", "error_E0.110_nu0.800_K0.100_a1.000_nx032_ne008_l005_centered_altgrad.npz")


def test_compute_once_then_load(tmp_path):
    calls = []

    def compute():
        calls.append(1)
        return {"err_l2_eta": np.arange(4.0), "rel_err_l2_p": np.float64(0.25)}
    name = results_filename(str(tmp_path / "sweep"), 1.0, 0.3, 0.1, 1.0, 16, 2, 1, "centered")
    a = cached_results(name, compute)
    b = cached_results(name, compute)
    assert len(calls) == 1 and os.path.exists(name)
    assert np.array_equal(a["err_l2_eta"], b["err_l2_eta"]) and float(b["rel_err_l2_p"]) == 0.25


def test_unreadable_file_is_recomputed(tmp_path):
    name = str(tmp_path / "bad.npz")
    with open(name, "wb") as fh:
        fh.write(b"not an npz")
    out = cached_results(name, lambda: {"x": np.ones(2)})
    assert np.array_equal(out["x"], np.ones(2)) and np.array_equal(np.load(name)["x"], np.ones(2))
