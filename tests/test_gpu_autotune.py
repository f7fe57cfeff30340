"""GEMM tile configurations and the autotuner.

Every FP64 tensor-core tile configuration, forced at all three GEMM call
sites, must reproduce the reference's nonlinear perturbation step (golden
fixture, relative L2 <= 1e-10). The autotuner must pick valid configurations
with measured times, and since all GEMM configurations sum over K in the same
order, a tuned plan must step bit-identically to an untuned one with the same
x-pass and split-TF32 kernels.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _plan(shape, lengths, re, dt, **kw):
    modes, phys = mode_counts(tuple(shape))
    return StepPlan(modes, phys, *lengths, _native.JSD_KIND_PERTURBATION, float(re), float(dt), linearise=False,
                    base_u=1 - cheb_points(modes[1]) ** 2, **kw)


def _steps(plan, u0, n):
    st = to_device_layout(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    plan.step(st, dp, 0, n)
    torch.cuda.synchronize()
    return st


@pytest.mark.parametrize("config", range(_native.DGEMM_CONFIGS))
def test_every_tile_configuration_matches_reference(cuda, config):
    d = golden("nonlin_pert_9x33x9")
    p = _plan(d["shape"], d["lengths"], d["re"], d["dt"])
    for site in _native.GEMM_SITES:
        p.set_gemm_config(site, config)
    assert all(c == config for c, _ in p.gemm_configs().values())
    st = _steps(p, d["u0"], 20)
    assert rel(to_reference_layout(st).cpu().numpy(), d["u20"]) < TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotuned_plan_steps_identically(cuda, precision):
    shape, lx, lz, re, dt = (48, 65, 48), 2 * np.pi, np.pi, 5000.0, 0.005
    u0 = seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-3, seed=3)
    plain = _plan(shape, (lx, lz), re, dt, precision=precision)
    tuned = _plan(shape, (lx, lz), re, dt, precision=precision, autotune=True)
    cfgs = tuned.gemm_configs()
    for site, (cfg, times) in cfgs.items():
        assert 0 <= cfg < _native.DGEMM_CONFIGS
        if precision == "mixed" and site == "dfield":
            continue  # the mixed form's y-derivatives do not use the DMMA kernel
        assert all(t > 0 for t in times)
        assert times[cfg] == min(times)
    # the kernel choices that change round-off (x-pass variant, split-TF32
    # kernel, eigenbasis kernel) are copied, so the plans differ only in GEMM
    # tiles, which never change a result
    plain.set_xmid_variant(tuned.xmid_variant()[0])
    if precision == "mixed":
        plain.set_split_kernel(tuned.split_kernel()[0])
        for site in (1, 2):
            plain.set_eig_kernel(site, tuned.eig_kernel(site)[0])
    a = _steps(plain, u0, 3)
    b = _steps(tuned, u0, 3)
    assert torch.equal(a, b)


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_every_xmid_variant_matches_reference(cuda, variant):
    """x-pass kernels (S-lane register FFT, half-split register FFT,
    shared-memory FFT) on the golden nonlinear perturbation case, FP64."""
    d = golden("nonlin_pert_9x33x9")
    p = _plan(d["shape"], d["lengths"], d["re"], d["dt"])
    p.set_xmid_variant(variant)
    assert p.xmid_variant()[0] == variant
    st = _steps(p, d["u0"], 20)
    assert rel(to_reference_layout(st).cpu().numpy(), d["u20"]) < TOL


def test_xmid_variants_agree_in_mixed_precision(cuda):
    shape, lx, lz, re, dt = (48, 65, 48), 2 * np.pi, np.pi, 5000.0, 0.005
    u0 = seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-3, seed=5)
    out = []
    for v in (0, 1, 2):
        p = _plan(shape, (lx, lz), re, dt, precision="mixed")
        p.set_xmid_variant(v)
        out.append(to_reference_layout(_steps(p, u0, 5)).cpu().numpy())
    assert rel(out[1], out[0]) < 1e-6 and rel(out[2], out[0]) < 1e-6


def test_autotune_chooses_an_available_xmid_variant(cuda):
    shape, lx, lz, re, dt = (48, 65, 48), 2 * np.pi, np.pi, 5000.0, 0.005
    p = _plan(shape, (lx, lz), re, dt, autotune=True)
    v, times = p.xmid_variant()
    assert times[v] > 0 and times[v] == min(t for t in times if t > 0)
