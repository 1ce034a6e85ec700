"""Checkpointing is not used by the fixtures."""


class CheckpointManagerOptions:
    def __init__(self, *_, **__):
        pass


class PyTreeCheckpointer:
    pass


class CheckpointManager:
    def __init__(self, *_, **__):
        raise NotImplementedError("orbax checkpoints are not provided by the stand-in")
