def shard_map(f, mesh=None, in_specs=None, out_specs=None, **_):
    """One device holds the whole array: the mapped function is the function."""
    return f
