"""ctypes binding of the native step library (libjsd.so, C ABI in include/jsd.h).

The library is built in-tree (``jax_spectral_dns/_build.py``) and loaded from
this package directory. There is no fallback: if the library is missing or
fails to load, every time-stepping call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libjsd.so")

JSD_KIND_NS = 0
JSD_KIND_PERTURBATION = 1
JSD_KIND_DUAL = 2

_dp = ctypes.POINTER(ctypes.c_double)


class JsdDesc(ctypes.Structure):
    """Mirror of ``jsd_desc`` (include/jsd.h)."""

    _fields_ = [
        ("mx", ctypes.c_int), ("ny", ctypes.c_int), ("mz", ctypes.c_int),
        ("px_ref", ctypes.c_int), ("pz_ref", ctypes.c_int),
        ("px_fft", ctypes.c_int), ("pz_fft", ctypes.c_int),
        ("lx", ctypes.c_double), ("lz", ctypes.c_double),
        ("kind", ctypes.c_int), ("linearise", ctypes.c_int), ("constant_mass_flux", ctypes.c_int),
        ("re_tau", ctypes.c_double), ("dt", ctypes.c_double), ("dt_explicit", ctypes.c_double),
        ("flow_rate_target", ctypes.c_double),
        ("base_u", _dp), ("base_du", _dp),
        ("D", _dp), ("V", _dp), ("Vinv", _dp), ("lam", _dp), ("sgn", _dp),
        ("c0", _dp), ("cN", _dp), ("w0", _dp), ("wN", _dp), ("y_weights", _dp),
        ("rhs_ns", _dp), ("lhs_inv_ns", _dp),
        ("precision", ctypes.c_int),
        ("n_batch", ctypes.c_int), ("re_tau_batch", _dp),
    ]


JSD_PRECISION_FP64 = 0
JSD_PRECISION_MIXED = 1


EXPORTED = (
    "jsd_plan_create", "jsd_plan_destroy", "jsd_step", "jsd_set_history", "jsd_set_source",
    "jsd_correct_mass_flux", "jsd_energy", "jsd_flow_rate", "jsd_nonlinear_terms",
    "jsd_workspace_bytes", "jsd_launches_per_step", "jsd_last_error", "jsd_abi_version",
    "jsd_profile_enable", "jsd_profile_read", "jsd_energy_noalloc", "jsd_step_trajectory",
    "jsd_launches_first_step_extra", "jsd_autotune", "jsd_gemm_config",
    "jsd_set_gemm_config", "jsd_xmid_variant", "jsd_set_xmid_variant",
    "jsd_energy_runs", "jsd_set_batch_active", "jsd_batch_active",
    "jsd_split_kernel", "jsd_set_split_kernel", "jsd_split_eig_in", "jsd_set_split_eig_in", "jsd_device_error",
    "jsd_set_coupling_term", "jsd_set_base_flow", "jsd_eig_kernel", "jsd_set_eig_kernel",
    "jsd_set_wait_limit", "jsd_wait_limit", "jsd_step_adjoint", "jsd_energy_grad",
)

ABI_VERSION = 5  # JSD_ABI_VERSION of include/jsd.h this binding is written for

# status codes (enum jsd_status)
JSD_ERR_ARG, JSD_ERR_CUDA, JSD_ERR_NOMEM, JSD_ERR_STATE, JSD_ERR_NONFINITE = -1, -2, -3, -4, -5

# GEMM call sites of a plan (jsd_gemm_config) and the number of DMMA tile configurations
GEMM_SITES = {"dfield": 0, "eig_in": 1, "eig_out": 2}
DGEMM_CONFIGS = 7

PROF_CLASSES = {"gemm": 0, "zinv": 1, "xmid": 2, "zfwd": 3, "eigen": 4, "linear": 5, "sgemm": 6}

_lib = None


class NativeError(RuntimeError):
    """A native call returned an error status (``code``: the JSD_ERR_* value)."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class DeviceFailure(NativeError):
    """The device reported a failure after the fact: a kernel's bounded wait
    expired (code JSD_ERR_CUDA) or the state became non-finite (code
    JSD_ERR_NONFINITE). Results since the last check are invalid."""


def load(path: str = LIB_PATH):
    """Load libjsd.so and declare its signatures (raises if it is absent)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise NativeError(
            f"native library not found at {path}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (requires nvcc)")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.jsd_plan_create.argtypes = [ctypes.POINTER(JsdDesc), ctypes.POINTER(vp)]
    lib.jsd_plan_destroy.argtypes = [vp]
    lib.jsd_step.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, vp]
    lib.jsd_set_history.argtypes = [vp, vp, ctypes.c_int]
    lib.jsd_set_source.argtypes = [vp, vp, vp, vp]
    lib.jsd_step_trajectory.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
    lib.jsd_correct_mass_flux.argtypes = [vp, vp, vp, vp]
    lib.jsd_energy.argtypes = [vp, vp, vp, vp]
    lib.jsd_flow_rate.argtypes = [vp, vp, vp, vp]
    lib.jsd_nonlinear_terms.argtypes = [vp, vp, ctypes.c_int, vp, vp, vp]
    lib.jsd_workspace_bytes.argtypes = [vp]
    lib.jsd_workspace_bytes.restype = ctypes.c_size_t
    lib.jsd_launches_per_step.argtypes = [vp]
    lib.jsd_launches_first_step_extra.argtypes = [vp]
    lib.jsd_last_error.restype = ctypes.c_char_p
    lib.jsd_energy_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, vp, vp, vp]
    lib.jsd_profile_enable.argtypes = [vp, ctypes.c_int]
    lib.jsd_autotune.argtypes = [vp, vp]
    lib.jsd_gemm_config.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    lib.jsd_set_gemm_config.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.jsd_xmid_variant.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    lib.jsd_energy_runs.argtypes = [vp, vp, vp, vp]
    lib.jsd_split_kernel.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    lib.jsd_set_split_kernel.argtypes = [vp, ctypes.c_int]
    lib.jsd_split_eig_in.argtypes = [vp]
    lib.jsd_set_split_eig_in.argtypes = [vp, ctypes.c_int]
    lib.jsd_eig_kernel.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    lib.jsd_set_eig_kernel.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.jsd_device_error.argtypes = [vp, vp]
    lib.jsd_set_wait_limit.argtypes = [vp, ctypes.c_int]
    lib.jsd_wait_limit.argtypes = [vp]
    lib.jsd_step_adjoint.argtypes = [vp, vp, ctypes.c_int, vp]
    lib.jsd_energy_grad.argtypes = [vp, vp, vp, vp]
    lib.jsd_set_coupling_term.argtypes = [vp, ctypes.c_int]
    lib.jsd_set_base_flow.argtypes = [vp, vp, vp, vp]
    lib.jsd_set_batch_active.argtypes = [vp, ctypes.c_int]
    lib.jsd_batch_active.argtypes = [vp]
    lib.jsd_set_xmid_variant.argtypes = [vp, ctypes.c_int]
    lib.jsd_profile_read.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)]
    for name in EXPORTED:
        if name not in ("jsd_workspace_bytes", "jsd_last_error"):
            getattr(lib, name).restype = ctypes.c_int
    if lib.jsd_abi_version() != ABI_VERSION:
        raise NativeError(f"{path} has ABI version {lib.jsd_abi_version()}, this binding needs {ABI_VERSION}; "
                          "rebuild it")
    if path == LIB_PATH:
        _lib = lib
    return lib


def check(rc: int, what: str, exc=NativeError):
    if rc != 0:
        msg = load().jsd_last_error().decode(errors="replace")
        raise exc(f"{what} failed ({rc}): {msg}", rc)
