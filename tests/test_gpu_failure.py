"""Device-side failure detection, exercised without faulting the GPU.

1. Non-finite state: a NaN is planted in the initial field on the host; after
   one step jsd_device_error reports JSD_ERR_NONFINITE (every stage checks the
   state it reconstructs), the flag is cleared by the read, and a clean field
   stepped next reports nothing. Covered for the FP64 form and for the mixed
   form on the tcgen05 kernels (the int8 eigenbasis products must carry the
   NaN through rather than slice it away).
2. Expired waits: the plan's wait limit is set to one poll, so the pipeline
   waits of the tcgen05 kernels give up on the first step; the kernels stop,
   wait for their own copies and MMAs in flight, free their tensor memory and
   return, and jsd_device_error reports JSD_ERR_CUDA. With the default limit
   restored the same plan steps the same field to the same result as a fresh
   plan, so the context and the plan stay usable.
The reference's own failure check is a host assert on the objective
(gradient_descent_solver.py:125).
"""
import numpy as np
import pytest
import torch

from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
LX, LZ, RE, DT = 2 * np.pi, np.pi, 4000.0, 0.005
SHAPE = (32, 65, 32)


def _plan(precision, tcgen05=False):
    modes, phys = mode_counts(SHAPE)
    p = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, RE, DT, linearise=False,
                 base_u=1 - cheb_points(modes[1]) ** 2, precision=precision)
    if tcgen05:
        p.set_split_kernel(1)
        for site in (1, 2):
            p.set_eig_kernel(site, 1)
    return p


def _field(seed=5):
    return seeded_velocity_hat(SHAPE, (LX, LZ), (6, 6), 1e-3, seed=seed)


def _step(plan, u0, n=1):
    st = to_device_layout(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    plan.step(st, dp, 0, n)
    torch.cuda.synchronize()
    return st


@pytest.mark.parametrize("precision,tcgen05", [("fp64", False), ("mixed", True)])
def test_nan_in_state_is_reported(cuda, precision, tcgen05):
    plan = _plan(precision, tcgen05)
    bad = _field().copy()
    bad[1, 3, 20, 2] = complex(np.nan, 0.0)  # one wall-normal velocity coefficient
    _step(plan, bad)
    with pytest.raises(_native.DeviceFailure) as e:
        plan.check_device_errors()
    assert e.value.code == _native.JSD_ERR_NONFINITE
    plan.check_device_errors()  # the read cleared the flag
    st = _step(plan, _field(), n=2)
    plan.check_device_errors()
    assert bool(torch.isfinite(torch.view_as_real(st)).all())


def test_infinity_in_state_is_reported(cuda):
    plan = _plan("mixed", tcgen05=True)
    bad = _field().copy()
    bad[0, 0, 10, 0] = complex(np.inf, 0.0)  # the mean flow
    _step(plan, bad)
    with pytest.raises(_native.DeviceFailure) as e:
        plan.check_device_errors()
    assert e.value.code == _native.JSD_ERR_NONFINITE


def test_expired_waits_are_reported_and_plan_recovers(cuda):
    u0 = _field(seed=9)
    plan = _plan("mixed", tcgen05=True)
    assert plan.wait_limit() == 1 << 22
    plan.set_wait_limit(1)
    assert plan.wait_limit() == 1
    _step(plan, u0)
    with pytest.raises(_native.DeviceFailure) as e:
        plan.check_device_errors()
    assert e.value.code == _native.JSD_ERR_CUDA
    plan.set_wait_limit(0)  # default again
    assert plan.wait_limit() == 1 << 22
    got = to_reference_layout(_step(plan, u0, n=3)).cpu().numpy()
    plan.check_device_errors()
    want = to_reference_layout(_step(_plan("mixed", tcgen05=True), u0, n=3)).cpu().numpy()
    np.testing.assert_array_equal(got, want)


def test_drop_in_step_raises_on_nonfinite_state(cuda):
    """The drop-in perform_time_step reads the flag before handing the result back."""
    from jax_spectral_dns.domain import PhysicalDomain
    from jax_spectral_dns.field import FourierField, VectorField
    from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation

    shape = (8, 33, 8)
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(LX, 1.0, LZ), aliasing=3 / 2)
    u0 = seeded_velocity_hat(shape, (LX, LZ), (3, 3), 1e-4, seed=1)
    vel = VectorField.FromData(FourierField, dom, torch.as_tensor(u0, device="cuda"), name="velocity_hat")
    nse = NavierStokesVelVortPerturbation(vel, Re=RE, dt=DT, end_time=10 * DT, linearise=False)
    bad = u0.copy()
    bad[2, 1, 5, 1] = complex(0.0, np.nan)
    with pytest.raises(_native.DeviceFailure):
        nse.perform_time_step(torch.as_tensor(bad, device="cuda"), 0.0, 0)
    out, _ = nse.perform_time_step(torch.as_tensor(u0, device="cuda"), 0.0, 0)
    assert bool(torch.isfinite(torch.view_as_real(out)).all())
