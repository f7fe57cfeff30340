"""The allocation-free energy entry point (jsd_energy_noalloc), through the C ABI.

It exists for callers that cannot allocate device memory (a host framework
that has reserved the GPU's memory for its own pool, or monitoring hooks in a
time loop that must not allocate). Its result must equal the plan-based
jsd_energy on the same state, on two consecutive calls (the shared static
scratch keeps the previous call's contents, which must not leak into the
next result). This file is collected last so a failure here comes after every
other test has run.
"""
import ctypes

import numpy as np
import pytest
import torch

from jax_spectral_dns import _native
from jax_spectral_dns._ops import operator_tables
from jax_spectral_dns._plan import StepPlan, to_device_layout
from jax_spectral_dns.seeds import mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _noalloc_energy(lib, state, modes, phys, lx, lz, weights):
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=state.device)
    rc = lib.jsd_energy_noalloc(ctypes.c_void_p(state.data_ptr()), modes[0], modes[1], modes[2], phys[0], phys[2],
                                lx, lz, ctypes.c_void_p(weights.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _native.check(rc, "jsd_energy_noalloc")
    torch.cuda.synchronize()
    return out.item()


def test_energy_noalloc_matches_plan_energy(cuda):
    lib = _native.load()
    shape, lx, lz = (32, 65, 32), 2 * np.pi, np.pi
    modes, phys = mode_counts(shape)
    weights = torch.as_tensor(operator_tables(modes[1]).y_weights, dtype=torch.float64, device=cuda)
    plan = StepPlan(modes, phys, lx, lz, 0, 180.0, 0.002)
    for seed, e0 in ((3, 1e-3), (4, 2.5e-2)):  # two calls in a row, different states
        st = to_device_layout(seeded_velocity_hat(shape, (lx, lz), (8, 8), e0, seed=seed), device=cuda)
        want = plan.energy(st).item()
        got = _noalloc_energy(lib, st, modes, phys, lx, lz, weights)
        assert abs(got / want - 1) < TOL, (seed, got, want)
        assert abs(got / e0 - 1) < 1e-10


def test_energy_noalloc_rejects_oversized_grid(cuda):
    lib = _native.load()
    dummy = torch.zeros(1, dtype=torch.float64, device=cuda)
    rc = lib.jsd_energy_noalloc(ctypes.c_void_p(dummy.data_ptr()), 3, 5000, 3, 4, 4, 1.0, 1.0,
                                ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()), None)
    assert rc == -1
    assert b"at most 4096" in lib.jsd_last_error()
