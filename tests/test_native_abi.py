"""The C-ABI library loads and exports every symbol include/jsd.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "jsd.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(jsd_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from jax_spectral_dns import _build, _native

    if not os.path.exists(_native.LIB_PATH):
        _build.build()
    return _native.load()


def test_header_declares_entry_points():
    names = _declared()
    for n in ("jsd_plan_create", "jsd_step", "jsd_energy", "jsd_set_history"):
        assert n in names


def test_every_declared_symbol_is_exported(lib):
    for name in _declared():
        assert hasattr(lib, name), name


def test_binding_covers_header(lib):
    from jax_spectral_dns import _native

    assert set(_declared()) <= set(_native.EXPORTED) | {"jsd_abi_version", "jsd_last_error"}


def test_abi_version_and_error_strings(lib):
    from jax_spectral_dns import _native

    assert lib.jsd_abi_version() == _native.ABI_VERSION == 5
    assert isinstance(lib.jsd_last_error(), bytes)


def test_status_codes_match_header():
    """The binding's status codes are the header's enum values."""
    from jax_spectral_dns import _native

    src = open(HEADER).read()
    codes = dict(re.findall(r"(JSD_ERR_[A-Z]+) = (-\d+)", src))
    assert "JSD_ERR_NONFINITE" in codes
    for name, val in codes.items():
        assert getattr(_native, name) == int(val), name


def test_wait_limit_argument_checks_without_gpu(lib):
    """jsd_set_wait_limit validates before touching a plan."""
    assert lib.jsd_set_wait_limit(None, 10) == -1
    assert lib.jsd_wait_limit(None) == 0


def test_set_source_argument_checks_without_gpu(lib):
    """jsd_set_source rejects a missing plan before touching it."""
    assert lib.jsd_set_source(None, None, None, None) == -1
    assert b"plan" in lib.jsd_last_error()


def test_plan_create_rejects_bad_descriptor_without_gpu(lib):
    """Argument validation happens before any CUDA call."""
    from jax_spectral_dns import _native

    d = _native.JsdDesc()
    d.mx, d.ny, d.mz = 4, 33, 9  # even mode count
    h = ctypes.c_void_p()
    rc = lib.jsd_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == -1
    assert b"odd" in lib.jsd_last_error()
