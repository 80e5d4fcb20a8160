"""jax.sharding stand-in: single device, no-op partitioning."""


class AxisType:
    Explicit = "explicit"
    Auto = "auto"


class PartitionSpec(tuple):
    def __new__(cls, *a):
        return tuple.__new__(cls, a)


class NamedSharding:
    def __init__(self, mesh, spec):
        self.mesh = mesh
        self.spec = spec


def reshard(x, spec):
    return x
