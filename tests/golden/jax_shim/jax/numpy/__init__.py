"""jax.numpy stand-in: NumPy plus a functional `.at[idx].set/get/add` indexer."""
import numpy as _np
from numpy import *  # noqa: F401,F403
from numpy import fft, linalg  # noqa: F401


class _AtIndex:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def set(self, value):
        out = _np.array(self.arr, copy=True)
        if _np.iscomplexobj(value) and not _np.iscomplexobj(out):
            out = out.astype(complex)
        out[self.idx] = value
        return out.view(A)

    def get(self):
        return _np.asarray(self.arr)[self.idx]

    def add(self, value):
        out = _np.array(self.arr, copy=True)
        out[self.idx] += value
        return out.view(A)


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self.arr, idx)


class A(_np.ndarray):
    @property
    def at(self):
        return _At(self)


def _wrap(fun):
    def wrapped(*args, **kwargs):
        res = fun(*args, **kwargs)
        return res.view(A) if isinstance(res, _np.ndarray) else res

    return wrapped


for _name in ["asarray", "zeros", "zeros_like", "ones", "ones_like", "concatenate",
              "moveaxis", "block", "flip", "take", "pad", "einsum", "split", "reshape",
              "insert", "stack", "meshgrid", "arange", "eye", "roll", "linspace"]:
    globals()[_name] = _wrap(getattr(_np, _name))


def array(x, dtype=None, **kwargs):
    return _np.array(x, dtype=dtype).view(A)


ndarray = _np.ndarray
