"""StepPlan.step_host_stream: host states stepped with their copies overlapped
(copy stream, two device buffers each way) give the same results as copying
each state in, stepping it and copying it back one after another."""
import numpy as np
import pytest
import torch

from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
SHAPE, LX, LZ = (16, 33, 16), 2 * np.pi, np.pi


@pytest.mark.parametrize("n_states", [1, 2, 5])
def test_host_stream_equals_one_by_one(cuda, n_states):
    modes, phys = mode_counts(SHAPE)
    plan = StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, 3000.0, 0.01, linearise=False,
                    base_u=1 - cheb_points(modes[1]) ** 2)
    states = [seeded_velocity_hat(SHAPE, (LX, LZ), (6, 6), 1e-3, seed=70 + k) for k in range(n_states)]
    host_in = [torch.as_tensor(u).pin_memory() for u in states]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    plan.step_host_stream(host_in, host_out, dp, 0, 3)
    torch.cuda.synchronize()
    plan.check_device_errors()
    for k, u in enumerate(states):
        st = to_device_layout(u)
        plan.step(st, torch.zeros(1, dtype=torch.float64, device="cuda"), 0, 3)
        want = to_reference_layout(st).cpu().numpy()
        np.testing.assert_array_equal(host_out[k].numpy(), want)
