"""``downsample_field`` (``src/utils.py:78-106``: ``jax.image.resize`` with the
antialiased bicubic method on every component) against the oracle's
restatement of JAX's published resize algorithm (``oracle/utils.py``), on the
host: the product's implementation is device-agnostic torch code."""
import numpy as np
import pytest
import torch

import oracle.utils as OU
from xlb_biot_b200.utils import downsample_field


@pytest.mark.parametrize("shape,factor", [((16, 12, 2), 2), ((30, 21, 3), 3), ((17, 13, 1), 4), ((64, 64, 2), 8)])
def test_matches_jax_resize_restatement(shape, factor):
    f = np.random.default_rng(sum(shape) + factor).standard_normal(shape)
    got = downsample_field(torch.as_tensor(f), factor).numpy()
    ref = OU.downsample_field(f, factor)
    assert got.shape == ref.shape == tuple(d // factor for d in shape[:-1]) + (shape[-1],)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_factor_one_is_identity_and_constants_are_kept():
    f = torch.randn(8, 6, 2, dtype=torch.float64)
    assert downsample_field(f, 1) is f
    c = torch.full((24, 18, 3), 2.5, dtype=torch.float64)
    assert torch.allclose(downsample_field(c, 3), torch.full((8, 6, 3), 2.5, dtype=torch.float64), atol=1e-13)


def test_weights_are_antialiased_keys_cubic():
    w = OU.weight_matrix(8, 4)                 # factor 2: kernel stretched by 2
    assert np.allclose(w.sum(axis=0), 1.0)
    # output 1 sits at input x = 2.5: taps |x - i| / 2 < 2, i.e. inputs 0..6
    k = OU.keys_cubic((np.arange(8) - 2.5) / 2.0)
    assert np.allclose(w[:, 1], k / k.sum())
    assert np.count_nonzero(w[:, 1]) == 7
