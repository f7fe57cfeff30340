"""Split-TF32 products on tcgen05 (k_tc05_split) in the mixed form: the
y-derivatives, and the eigenbasis-in products of the nonlinear terms.

The tcgen05 kernel (accumulator in tensor memory) must agree with the
mma.sync split kernel to FP32-accumulation level and with the FP64 form to the
mixed form's own level, for Ny <= 128 and for Ny = 129 (the y = -1 wall row
in FP64 beside the 128-row tensor part); its bounded waits must never expire.
Splitting the eigenbasis-in products (their inputs come out of FP32
transforms and products) must leave the state at the same level as
FP64-accurate products of the same terms.
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


def _plan(shape, precision):
    modes, phys = mode_counts(shape)
    return StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT, linearise=False,
                    base_u=1 - cheb_points(modes[1]) ** 2, precision=precision)


def _run(plan, u0, n):
    st = to_device_layout(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    plan.step(st, dp, 0, n)
    torch.cuda.synchronize()
    return to_reference_layout(st).cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 65, 16), (16, 129, 16), (32, 97, 16)])
def test_tcgen05_split_kernel(cuda, shape):
    u0 = seeded_velocity_hat(shape, (LX, LZ), (6, 6), 1e-3, seed=11)
    a = _plan(shape, "mixed")
    a.set_split_kernel(1)  # small boxes start on k_sgemm3; the tcgen05 kernel is selectable
    out_tc = _run(a, u0, 6)
    a.check_device_errors()
    b = _plan(shape, "mixed")
    b.set_split_kernel(0)
    out_mma = _run(b, u0, 6)
    out_64 = _run(_plan(shape, "fp64"), u0, 6)
    assert rel(out_tc, out_mma) < 1e-6
    assert rel(out_tc, out_64) < 1e-5
    # nonlinear terms of the first stage (all rows through the chosen kernel)
    st = to_device_layout(u0)
    hv_a, hg_a = a.nonlinear_terms(st)
    hv_b, hg_b = b.nonlinear_terms(st)
    assert rel(hv_a.cpu().numpy(), hv_b.cpu().numpy()) < 1e-5 and rel(hg_a.cpu().numpy(), hg_b.cpu().numpy()) < 1e-5
    a.check_device_errors()


@pytest.mark.parametrize("shape", [(16, 65, 16), (16, 129, 16), (32, 97, 16)])
@pytest.mark.parametrize("kernel", [0, 1])
def test_split_eigenbasis_in(cuda, shape, kernel):
    """V^-1 D q, V^-1 H1, V^-1 h_g in split TF32 (two operators in one
    tcgen05 launch; the mixed default without a base flow, selected here for a
    perturbation plan) against FP64-accurate products."""
    u0 = seeded_velocity_hat(shape, (LX, LZ), (6, 6), 1e-3, seed=12)
    a = _plan(shape, "mixed")
    a.set_split_kernel(kernel)
    assert a.split_eig_in() == 0  # the default with a base flow
    a.set_split_eig_in(True)
    assert a.split_eig_in() == 1
    out_split = _run(a, u0, 6)
    a.check_device_errors()
    b = _plan(shape, "mixed")
    b.set_split_kernel(kernel)
    b.set_split_eig_in(False)
    assert b.split_eig_in() == 0
    out_exact = _run(b, u0, 6)
    out_64 = _run(_plan(shape, "fp64"), u0, 6)
    assert rel(out_split, out_exact) < 1e-6
    assert rel(out_split, out_64) < 1e-5
    assert _plan(shape, "fp64").split_eig_in() == -1


def test_autotune_picks_a_split_kernel(cuda):
    modes, phys = mode_counts((32, 129, 32))
    p = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT, base_u=1 - cheb_points(129) ** 2,
                 precision="mixed", autotune=True)
    k, times = p.split_kernel()
    assert k in (0, 1) and all(t > 0 for t in times) and times[k] == min(times)
    p.check_device_errors()
    with pytest.raises(_native.NativeError):
        _plan((16, 65, 16), "fp64").set_split_kernel(1)
