"""NumPy-backed stand-in for the subset of the jax API that the reference solver uses.

JAX is not installed in this environment. ``make_golden.py`` puts this directory first on
``sys.path`` so that the reference's own Python solver
(``src/jaxmaterials/solver/lippmann_schwinger.py``) can be imported and executed
unchanged, with NumPy doing the arithmetic in the same dtypes (float32 stays float32,
complex64 FFTs for float32 input). Only the calls that solver makes are provided.
"""

from . import numpy  # noqa: F401
from . import lax  # noqa: F401


class _Config:
    def update(self, *args, **kwargs):
        pass


config = _Config()


def jit(fun=None, **kwargs):
    """No tracing: return the function itself (also usable as ``jit(static_argnames=..)``)."""
    if fun is None:
        return lambda f: f
    return fun
