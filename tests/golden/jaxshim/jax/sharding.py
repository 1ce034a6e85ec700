"""Sharding types of ``jax.sharding``: inert on one device."""


class PartitionSpec(tuple):
    def __new__(cls, *parts):
        return tuple.__new__(cls, parts)


class Mesh:
    def __init__(self, devices, axis_names):
        self.devices, self.axis_names = devices, axis_names


class NamedSharding:
    def __init__(self, mesh, spec):
        self.mesh, self.spec = mesh, spec


class PositionalSharding:
    def __init__(self, devices):
        self.devices = devices

    def reshape(self, *shape):
        return self
