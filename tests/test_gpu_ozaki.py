"""FP64-accurate eigenbasis products on the int8 tensor cores (k_oz8_gemm,
Ozaki splitting) in the mixed form.

Switched per call site against the FP64 DMMA kernel inside the same mixed
plan, only the eigenbasis products' round-off differs, so the states must
agree to FP64 level (a TF32- or FP32-level product would differ by ~1e-7);
against the FP64 form the plan stays at the mixed form's own level. Covers
the 129th row (V, D V at Ny = 129) and 129th column (V^-1 D) applied in FP64
beside the tensor part, even and odd Ny, and the bounded waits.
"""
import numpy as np
import pytest
import torch

from conftest import rel
from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
LX, LZ, RE, DT = 2 * np.pi, np.pi, 4000.0, 0.005
SITES = (1, 2)  # eigenbasis in, eigenbasis out


def _plan(shape, precision, kind=_native.JSD_KIND_PERTURBATION):
    modes, phys = mode_counts(shape)
    return StepPlan(modes, phys, LX, LZ, kind, RE, DT, linearise=False,
                    base_u=1 - cheb_points(modes[1]) ** 2, precision=precision)


def _run(plan, u0, n):
    st = to_device_layout(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    plan.step(st, dp, 0, n)
    torch.cuda.synchronize()
    return to_reference_layout(st).cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 129, 16), (16, 65, 16), (8, 24, 12), (32, 97, 32)])
def test_ozaki_eigen_products_are_fp64_accurate(cuda, shape):
    u0 = seeded_velocity_hat(shape, (LX, LZ), (6, 6), 1e-3, seed=21)
    oz = _plan(shape, "mixed")
    for site in SITES:
        oz.set_eig_kernel(site, 1)
        assert oz.eig_kernel(site)[0] == 1
    out_oz = _run(oz, u0, 3)
    oz.check_device_errors()
    dm = _plan(shape, "mixed")
    for site in SITES:
        dm.set_eig_kernel(site, 0)
    out_dm = _run(dm, u0, 3)
    assert rel(out_oz, out_dm) < 1e-11
    out_64 = _run(_plan(shape, "fp64"), u0, 3)
    assert rel(out_oz, out_64) < 1e-5


def test_ozaki_one_site_at_a_time(cuda):
    shape = (16, 129, 16)
    u0 = seeded_velocity_hat(shape, (LX, LZ), (6, 6), 1e-3, seed=22)
    ref = _plan(shape, "mixed")
    for site in SITES:
        ref.set_eig_kernel(site, 0)
    out_ref = _run(ref, u0, 2)
    for site in SITES:
        p = _plan(shape, "mixed")
        for s in SITES:
            p.set_eig_kernel(s, 1 if s == site else 0)
        assert rel(_run(p, u0, 2), out_ref) < 1e-11, site
        p.check_device_errors()


def test_ozaki_autotune_and_availability(cuda):
    modes, phys = mode_counts((32, 129, 32))
    p = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT, base_u=1 - cheb_points(129) ** 2,
                 precision="mixed", autotune=True)
    for site in SITES:
        k, times = p.eig_kernel(site)
        assert k in (0, 1) and all(t > 0 for t in times) and times[k] == min(times)
    p.check_device_errors()
    with pytest.raises(_native.NativeError):
        _plan((16, 65, 16), "fp64").set_eig_kernel(1, 1)
    with pytest.raises(_native.NativeError):
        _plan((16, 65, 16), "mixed").set_eig_kernel(0, 1)
