from . import tvd  # noqa: F401
