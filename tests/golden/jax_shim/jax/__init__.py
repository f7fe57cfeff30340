"""NumPy stand-in for the parts of `jax` the reference uses (test fixtures only).

jit/checkpoint are identities, lax control flow runs eagerly in Python, and
jax.numpy is NumPy with an `.at[]` indexer. Everything computes in float64.
"""
import numpy as _np

from . import numpy  # noqa: F401
from . import scipy  # noqa: F401


class _Config:
    def update(self, *args, **kwargs):
        pass


config = _Config()


def jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def checkpoint(fun, **kwargs):
    return fun


def grad(fun, argnums=0):
    """Derivative of a scalar real-analytic function by the complex step
    f'(x) = Im f(x + i h) / h (h = 1e-30): exact to round-off, no subtraction."""
    if argnums != 0:
        raise NotImplementedError("grad: only argnums=0")

    def d(x, *args):
        h = 1e-30
        return _np.imag(fun(x + 1j * h, *args)) / h

    return d


def default_backend():
    return "cpu"


def clear_caches():
    pass


def devices():
    return ["cpu"]


local_devices = devices


def _stack_tree(items):
    if isinstance(items[0], tuple):
        return tuple(_stack_tree([it[i] for it in items]) for i in range(len(items[0])))
    return _np.array(items).view(numpy.A)


class lax:
    @staticmethod
    def cond(pred, true_fun, false_fun, *operands):
        return true_fun(*operands) if pred else false_fun(*operands)

    @staticmethod
    def map(fun, xs, batch_size=None):
        # outputs stacked per leaf, as jax.lax.map does for tuple (pytree) results
        return _stack_tree([fun(x) for x in xs])

    @staticmethod
    def scan(fun, init, xs=None, length=None, **kwargs):
        carry = init
        ys = []
        n = length if xs is None else len(xs)
        for i in range(n):
            carry, y = fun(carry, None if xs is None else xs[i])
            ys.append(y)
        if ys and ys[0] is not None:
            return carry, _stack_tree(ys)
        return carry, None


class debug:
    @staticmethod
    def print(*args, **kwargs):
        pass

    @staticmethod
    def callback(fun, *args, **kwargs):
        fun(*args)
