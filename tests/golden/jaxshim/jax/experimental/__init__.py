from . import mesh_utils, multihost_utils, shard_map  # noqa: F401
