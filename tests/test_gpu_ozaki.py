"""FP64-accurate eigenbasis products on the int8 tensor cores (k_oz8_gemm,
Ozaki splitting).

In an FP64 plan the kernel replaces only the eigenbasis products, so with it
switched in the plan must still meet the reference fixtures at the parity
tolerance and agree with the DMMA products to FP64 round-off (a TF32- or
FP32-level product would miss both by orders of magnitude); in a mixed plan
the FP32 transforms amplify round-off differences, so there the bound is the
mixed form's. Covers the 129th row (V, D V at Ny = 129) and 129th column
(V^-1 D) applied in FP64 beside the tensor part, even and odd Ny, each site
alone, the autotuner's choice and the bounded waits.
"""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
LX, LZ, RE, DT = 2 * np.pi, np.pi, 4000.0, 0.005
SITES = (1, 2)  # eigenbasis in, eigenbasis out


def _plan(shape, precision, eig=0):
    modes, phys = mode_counts(shape)
    p = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT, linearise=False,
                 base_u=1 - cheb_points(modes[1]) ** 2, precision=precision)
    for site in SITES:
        p.set_eig_kernel(site, eig)
    return p


def _run(plan, u0, n):
    st = to_device_layout(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    plan.step(st, dp, 0, n)
    torch.cuda.synchronize()
    return to_reference_layout(st).cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 129, 16), (16, 65, 16), (8, 24, 12), (32, 97, 32)])
def test_ozaki_eigen_products_are_fp64_accurate(cuda, shape):
    u0 = seeded_velocity_hat(shape, (LX, LZ), (6, 6), 1e-3, seed=21)
    oz64 = _plan(shape, "fp64", eig=1)
    assert all(oz64.eig_kernel(site)[0] == 1 for site in SITES)
    out_oz64 = _run(oz64, u0, 3)
    oz64.check_device_errors()
    out_64 = _run(_plan(shape, "fp64"), u0, 3)
    assert rel(out_oz64, out_64) < 1e-12
    oz = _plan(shape, "mixed", eig=1)
    out_oz = _run(oz, u0, 3)
    oz.check_device_errors()
    assert rel(out_oz, _run(_plan(shape, "mixed"), u0, 3)) < 1e-7
    assert rel(out_oz, out_64) < 1e-5


def test_ozaki_fp64_plan_meets_reference_fixture(cuda):
    d = golden("nonlin_pert_9x33x9")
    shape = tuple(int(x) for x in d["shape"])
    modes, phys = mode_counts(shape)
    p = StepPlan(modes, phys, *d["lengths"], _native.JSD_KIND_PERTURBATION, float(d["re"]), float(d["dt"]),
                 linearise=False, base_u=1 - cheb_points(modes[1]) ** 2)
    for site in SITES:
        p.set_eig_kernel(site, 1)
    st = to_device_layout(d["u0"])
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    p.step(st, dp, 0, 20)
    assert rel(to_reference_layout(st).cpu().numpy(), d["u20"]) < 1e-10
    p.check_device_errors()


def test_ozaki_one_site_at_a_time(cuda):
    shape = (16, 129, 16)
    u0 = seeded_velocity_hat(shape, (LX, LZ), (6, 6), 1e-3, seed=22)
    out_ref = _run(_plan(shape, "fp64"), u0, 2)
    for site in SITES:
        p = _plan(shape, "fp64")
        p.set_eig_kernel(site, 1)
        assert rel(_run(p, u0, 2), out_ref) < 1e-12, site
        p.check_device_errors()


def test_ozaki_autotune_and_availability(cuda):
    modes, phys = mode_counts((32, 129, 32))
    p = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT, base_u=1 - cheb_points(129) ** 2,
                 precision="mixed", autotune=True)
    for site in SITES:
        k, times = p.eig_kernel(site)
        assert k in (0, 1) and all(t > 0 for t in times) and times[k] == min(times)
    p.check_device_errors()
    q = _plan((16, 65, 16), "fp64")
    assert all(q.eig_kernel(site)[0] == 0 for site in SITES)  # FP64 plans default to DMMA
    for shape, start in (((16, 65, 16), 0), ((100, 33, 100), 1)):
        modes, phys = mode_counts(shape)
        m = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT,
                     base_u=1 - cheb_points(modes[1]) ** 2, precision="mixed")
        # mixed plans start on the int8 kernel where each call has >= 8 tiles per SM
        assert all(m.eig_kernel(site)[0] == start for site in SITES), shape
        assert m.split_kernel()[0] == start, shape
    with pytest.raises(_native.NativeError):
        q.set_eig_kernel(0, 1)  # the y-derivative site has no int8 form
    with pytest.raises(_native.NativeError):
        _plan((8, 161, 8), "fp64").set_eig_kernel(1, 1)  # beyond 129 Chebyshev points
