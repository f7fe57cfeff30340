"""FP64 parity at the sizes of the benchmark configurations, against the
reference run under the NumPy shim (tests/golden/config1_49x65x49.npz: 100
nonlinear steps, config2_dual_33x65x33.npz, config4_129x129x129.npz: 3
channel steps, all from make_golden.py): the seeded input is rebuilt
here from the same seed helper, and each large state is compared through a
fixed seeded sample of 4096 entries plus its full norm, so the fixtures stay
small while every part of the state can be reached."""
import numpy as np
import pytest
import torch

from conftest import golden
from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.field import FourierField, VectorField
from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation
from jax_spectral_dns.navier_stokes_perturbation_dual import NavierStokesVelVortPerturbationDual
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _check(full, d, key, tol=TOL):
    """Sampled entries and the norm of `full` against the fixture's."""
    flat = np.asarray(full).ravel()
    sample = d[key + "_sample"]
    assert np.linalg.norm(flat[d["idx"]] - sample) < tol * np.linalg.norm(sample), key
    assert abs(np.linalg.norm(flat) / float(d[key + "_norm"]) - 1) < tol, key


def _seed(d):
    shape, (lx, lz) = tuple(int(x) for x in d["shape"]), d["lengths"]
    u0 = seeded_velocity_hat(shape, (lx, lz), tuple(int(k) for k in d["kmax"]), float(d["e0"]), seed=int(d["seed"]))
    _check(u0, d, "u0", 1e-14)  # the seed helper rebuilds the reference's input
    return shape, lx, lz, u0


def test_nonlinear_perturbation_at_config1_size(cuda):
    """49x65x49 modes, Re = 5000, dt = 0.005: 100 steps against the reference,
    the state after 1, 10, 50 and 100 steps and the energy after every step."""
    d = golden("config1_49x65x49")
    shape, lx, lz, u0 = _seed(d)
    modes, phys = mode_counts(shape)
    plan = StepPlan(modes, phys, lx, lz, _native.JSD_KIND_PERTURBATION, float(d["re"]), float(d["dt"]),
                    linearise=False, base_u=1 - cheb_points(modes[1]) ** 2)
    st = to_device_layout(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    energies = [plan.energy(st)]
    n = int(d["n_steps"])
    kept = {int(k) for k in d["kept_steps"]}
    assert n == 100 and kept == {1, 10, 50, 100}
    for t in range(n):
        plan.step(st, dp, t, 1)
        energies.append(plan.energy(st))
        if t + 1 in kept:
            _check(to_reference_layout(st).cpu().numpy(), d, f"u{t + 1}")
    plan.check_device_errors()
    np.testing.assert_allclose(torch.cat(energies).cpu().numpy(), d["energy"], rtol=TOL, atol=0)


def test_dual_gradient_at_config2_size(cuda):
    """33x65x33 modes, Re = 3000, T = 0.5: the drop-in dual class's gradient
    and gain against the reference dual solver's."""
    d = golden("config2_dual_33x65x33")
    shape, lx, lz, u0 = _seed(d)
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz), aliasing=3 / 2)
    vf = VectorField.FromData(FourierField, dom, torch.as_tensor(u0, device="cuda"), name="velocity_hat")
    n, dt = int(d["n_steps"]), float(d["dt"])
    nse = NavierStokesVelVortPerturbation(vf, Re=float(d["re"]), dt=dt, end_time=n * dt, linearise=True)
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
    grad = dual.get_grad().cpu().numpy()
    _check(grad, d, "grad")
    assert abs(dual.gain / float(d["gain"]) - 1) < TOL


def test_channel_step_at_benchmark_size(cuda):
    """The benchmark workload (129x129x129 modes, constant mass flux, Re_tau =
    180, dt = 0.002, bench.py's seeded field): three steps against the
    reference's own steps, through the fixture's sample and norm after steps
    1 and 3, with dPdx, the flow-rate target and the energy after every step."""
    from jax_spectral_dns.seeds import turbulent_channel_hat

    d = golden("config4_129x129x129")
    shape, (lx, lz) = tuple(int(x) for x in d["shape"]), d["lengths"]
    re_tau, dt = float(d["re_tau"]), float(d["dt"])
    u0 = turbulent_channel_hat(shape, (lx, lz), re_tau, tuple(int(k) for k in d["kmax"]), seed=int(d["seed"]))
    _check(u0, d, "u0", 1e-14)
    modes, phys = mode_counts(shape)
    probe = StepPlan(modes, phys, lx, lz, 0, re_tau, dt)
    q0 = probe.flow_rate(to_device_layout(u0)[0]).item()
    assert abs(q0 / float(d["flow_rate"]) - 1) < 1e-13
    del probe
    p = StepPlan(modes, phys, lx, lz, 0, re_tau, dt, constant_mass_flux=True, flow_rate_target=q0)
    st = to_device_layout(u0)
    dp = torch.full((1,), float(d["dpdx"][0]), dtype=torch.float64, device="cuda")
    assert int(d["n_steps"]) == 3
    for t in range(3):
        p.step(st, dp, t, 1)
        if t + 1 in (1, 3):
            _check(to_reference_layout(st).cpu().numpy(), d, f"u{t + 1}")
        want_dp = float(d["dpdx"][t + 1])
        assert abs(dp.item() - want_dp) < 1e-8 * max(1.0, abs(want_dp))
        assert abs(p.energy(st).item() / float(d["energy"][t + 1]) - 1) < TOL
    p.check_device_errors()
