import numpy as _np


def create_device_mesh(shape, *_, **__):
    return _np.array(["cpu:0"], dtype=object).reshape(shape)
