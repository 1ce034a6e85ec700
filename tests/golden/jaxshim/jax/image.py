"""``jax.image.resize`` is imported by the reference's ``src/utils.py`` (its
``downsample_field``); the fixtures do not call it."""


def resize(*_, **__):
    raise NotImplementedError("jax.image.resize is not provided by the stand-in")
