"""``jax.numpy`` subset on top of NumPy, with functional ``.at[...].set``."""

import numpy as _np

float32 = _np.float32
float64 = _np.float64


class _AtIndex:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def set(self, value):
        out = _np.array(self._arr, copy=True).view(JArray)
        out[self._idx] = value
        return out


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self._arr, idx)


class JArray(_np.ndarray):
    """ndarray with jax's functional update syntax ``a.at[i].set(v)``."""

    @property
    def at(self):
        return _At(self)


def _wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, JArray):
        return x.view(JArray)
    return x


def _axis(axis):
    return tuple(axis) if isinstance(axis, list) else axis


def _f(name):
    fn = getattr(_np, name)

    def g(*args, **kwargs):
        return _wrap(fn(*args, **kwargs))

    g.__name__ = name
    return g


for _name in ["zeros", "eye", "stack", "expand_dims", "sqrt", "abs", "real", "roll",
              "einsum", "dot", "array", "asarray", "ones", "ones_like", "zeros_like",
              "maximum", "minimum", "concatenate", "meshgrid", "exp", "sin", "cos"]:
    globals()[_name] = _f(_name)


def sum(a, axis=None, **kw):
    return _wrap(_np.sum(a, axis=_axis(axis), **kw))


def mean(a, axis=None, **kw):
    return _wrap(_np.mean(a, axis=_axis(axis), **kw))


def min(a, axis=None):
    return _wrap(_np.min(a, axis=_axis(axis)))


def max(a, axis=None):
    return _wrap(_np.max(a, axis=_axis(axis)))


def trace(a, axis1=0, axis2=1):
    return _wrap(_np.trace(a, axis1=axis1, axis2=axis2))


def where(cond, x, y):
    return _wrap(_np.where(cond, x, y))


def astype(a, dtype):
    return _wrap(_np.asarray(a).astype(dtype))


class _Fft:
    @staticmethod
    def fftn(a, axes=None):
        return _wrap(_np.fft.fftn(a, axes=axes))

    @staticmethod
    def ifftn(a, axes=None):
        return _wrap(_np.fft.ifftn(a, axes=axes))


class _Linalg:
    @staticmethod
    def solve(a, b):
        return _wrap(_np.linalg.solve(a, b))

    @staticmethod
    def eigh(a):
        return _np.linalg.eigh(a)

    @staticmethod
    def eigvalsh(a):
        return _wrap(_np.linalg.eigvalsh(a))

    @staticmethod
    def norm(a):
        return _wrap(_np.linalg.norm(a))


fft = _Fft()
linalg = _Linalg()
