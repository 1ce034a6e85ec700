"""Test infrastructure (CPU oracle): ``downsample_field`` of the reference
(``src/utils.py:78-106``), which resizes every component with
``jax.image.resize(..., method='bicubic')``.

JAX 0.5.3 (the version the reference pins, ``setup.sh``) is absent here, so its
published resize algorithm is restated (``jax/_src/image/scale.py``:
``scale_and_translate`` over each resized axis, ``compute_weight_mat`` with
``antialias=True``, Keys' cubic kernel with a = -0.5):

* output sample j of an axis scaled by s = n_out / n_in sits at input
  coordinate x_j = (j + 1/2) / s - 1/2;
* the kernel is stretched by max(1/s, 1) when downsampling (antialiasing);
* input i weighs k(|x_j - i| / stretch), weights normalised to sum 1 per
  output sample (a sum below 1000 * FP32 epsilon gives weight 0), and an
  output sample whose x_j lies outside [-1/2, n_in - 1/2] gets weight 0;
* axes are resized one after the other (separable).
"""
import numpy as np


def keys_cubic(x):
    """Keys' cubic convolution kernel, a = -0.5."""
    x = np.abs(x)
    return np.where(x < 1.0, ((1.5 * x - 2.5) * x) * x + 1.0,
                    np.where(x < 2.0, ((-0.5 * x + 2.5) * x - 4.0) * x + 2.0, 0.0))


def weight_matrix(n_in, n_out):
    """(n_in, n_out) weights of one axis, as ``compute_weight_mat``."""
    scale = n_out / n_in
    inv = 1.0 / scale
    stretch = max(inv, 1.0)
    sample = (np.arange(n_out) + 0.5) * inv - 0.5
    w = keys_cubic(np.abs(sample[None, :] - np.arange(n_in)[:, None]) / stretch)
    total = w.sum(axis=0, keepdims=True)
    w = np.where(np.abs(total) > 1000.0 * float(np.finfo(np.float32).eps),
                 w / np.where(total != 0, total, 1), 0.0)
    inside = (sample >= -0.5) & (sample <= n_in - 0.5)
    return np.where(inside[None, :], w, 0.0)


def image_resize_bicubic(image, shape):
    """``jax.image.resize(image, shape, 'bicubic')`` for 2-D images."""
    out = np.asarray(image, dtype=np.float64)
    for axis, n_out in enumerate(shape):
        n_in = out.shape[axis]
        if n_in == n_out:
            continue
        out = np.moveaxis(np.tensordot(out, weight_matrix(n_in, n_out), axes=([axis], [0])), -1, axis)
    return out


def downsample_field(field, factor, method='bicubic'):
    """``src/utils.py:78-106``."""
    if factor == 1:
        return field
    field = np.asarray(field, dtype=np.float64)
    new_shape = tuple(d // factor for d in field.shape[:-1])
    return np.stack([image_resize_bicubic(field[..., i], new_shape) for i in range(field.shape[-1])], axis=-1)
