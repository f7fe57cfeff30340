"""Optimal transient growth through the B200 linearised perturbation step:
the reference's test_transient_growth (tests/test_project.py:1489-1503) with
run_transient_growth's setup (examples.py:1274-1413): 5x50x5 modes, box
2 pi / alpha x 2 x 1e-3, dt = 0.01, the LinearStabilityCalculation optimal
initial field scaled to E0 = 1e-10. The DNS gain E(T) / E(0) must equal the
predicted optimal gain; the reference accepts 8e-4 (Re 600) and 3e-5
(Re 3000), the oracle's step reaches ~2e-7, and so must the device step."""
import math

import pytest

from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.linear_stability_calculation import LinearStabilityCalculation
from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("re,t", [(600.0, 2.0), (3000.0, 15.0)])
def test_transient_growth(cuda, re, t):
    alpha = 1.0
    dom = PhysicalDomain.create((4, 50, 4), (True, False, True),
                                scale_factors=(2 * math.pi / alpha, 1.0, 1.0e-3), aliasing=3 / 2)
    lsc = LinearStabilityCalculation(Re=re, alpha=alpha, beta=0.0, n=50)
    u = lsc.calculate_transient_growth_initial_condition(dom, t, 60, recompute_full=True)
    u_hat = (u * (1e-5 / math.sqrt(u.energy()))).hat()
    nse = NavierStokesVelVortPerturbation(u_hat, Re=re, dt=0.01, end_time=t, linearise=True)
    nse.activate_jit()
    nse.solve()
    e0 = nse.get_initial_field("velocity_hat").no_hat().energy()
    e_t = nse.get_latest_field("velocity_hat").no_hat().energy()
    e_max = lsc.calculate_transient_growth_max_energy(t, 60)
    assert abs((e_t / e0) / e_max - 1) < 1e-6
