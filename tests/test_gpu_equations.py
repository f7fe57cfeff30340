"""The drop-in equation classes (reference surface) on the GPU."""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.field import FourierField, VectorField
from jax_spectral_dns.navier_stokes import NavierStokesVelVort
from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation
from jax_spectral_dns.navier_stokes_perturbation_dual import NavierStokesVelVortPerturbationDual

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _vf(d):
    shape, (lx, lz) = tuple(d["shape"]), d["lengths"]
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz), aliasing=3 / 2)
    return VectorField.FromData(FourierField, dom, torch.as_tensor(d["u0"], device="cuda"), name="velocity_hat")


def test_perturbation_perform_time_step(cuda):
    d = golden("nonlin_pert_9x33x9")
    nse = NavierStokesVelVortPerturbation(_vf(d), Re=float(d["re"]), dt=float(d["dt"]), end_time=20 * float(d["dt"]),
                                          linearise=False)
    u = nse.get_initial_field("velocity_hat").get_data()
    dpdx = 0.0
    for t in range(20):
        u, dpdx = nse.perform_time_step(u, dpdx, t)
        if t == 0:
            assert rel(u.cpu().numpy(), d["u1"]) < TOL
    assert rel(u.cpu().numpy(), d["u20"]) < TOL


def test_perturbation_solve(cuda):
    d = golden("lin_pert_9x65x5")
    nse = NavierStokesVelVortPerturbation(_vf(d), Re=float(d["re"]), dt=float(d["dt"]), end_time=100 * float(d["dt"]),
                                          linearise=True)
    nse.activate_jit()
    nse.solve()
    uT = nse.get_latest_field("velocity_hat")
    assert rel(uT.get_data().cpu().numpy(), d["u100"]) < TOL
    assert abs(uT.no_hat().energy() / d["energy"][100] - 1) < 1e-10


def test_navier_stokes_constant_mass_flux_class(cuda):
    d = golden("ns_cmf_9x33x9")
    nse = NavierStokesVelVort(_vf(d), Re_tau=float(d["re_tau"]), dt=float(d["dt"]), end_time=10 * float(d["dt"]),
                              constant_mass_flux=True)
    assert abs(nse.flow_rate / float(d["flow_rate"]) - 1) < 1e-13
    assert abs(nse.dPdx - d["dpdx"][0]) < 1e-12 * abs(d["dpdx"][0])
    u, dpdx = nse.get_initial_field("velocity_hat").get_data(), nse.dPdx
    for t in range(10):
        u, dpdx = nse.perform_time_step(u, dpdx, t)
    assert rel(u.cpu().numpy(), d["u10"]) < TOL
    assert abs(dpdx - d["dpdx"][-1]) < 1e-8 * abs(d["dpdx"][-1])


def test_dual_class_gradient(cuda):
    d = golden("dual_lin_5x33x5")
    n, dt = int(d["n_steps"]), float(d["dt"])
    nse = NavierStokesVelVortPerturbation(_vf(d), Re=float(d["re"]), dt=dt, end_time=n * dt, linearise=True)
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
    grad = dual.get_grad()
    assert rel(grad.cpu().numpy(), d["grad"]) < TOL
    assert abs(dual.gain / float(d["gain"]) - 1) < TOL
    pg, ok = dual.get_projected_grad(1e-2)
    assert ok and bool(torch.isfinite(torch.view_as_real(pg)).all())


def test_dual_class_nonlinear_gradient(cuda):
    d = golden("dual_nonlin_9x33x9")
    n, dt = int(d["n_steps"]), float(d["dt"])
    nse = NavierStokesVelVortPerturbation(_vf(d), Re=float(d["re"]), dt=dt, end_time=n * dt, linearise=False)
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
    grad = dual.get_grad()
    assert rel(grad.cpu().numpy(), d["grad"]) < TOL
    assert abs(dual.gain / float(d["gain"]) - 1) < TOL


def test_instationary_base_flow_matches_reference(cuda):
    """NavierStokesVelVortPerturbationInstationary: base re-evaluated every
    step, coupling term off (reference fixture)."""
    from jax_spectral_dns.navier_stokes_perturbation_instationary import NavierStokesVelVortPerturbationInstationary

    d = golden("instationary_9x33x9")
    n, dt = int(d["n_steps"]), float(d["dt"])
    nse = NavierStokesVelVortPerturbationInstationary(_vf(d), Re=float(d["re"]), dt=dt, end_time=n * dt,
                                                      kappa=float(d["kappa"]), accelerate=True, n_max=int(d["n_max"]))
    u = nse.get_initial_field("velocity_hat").get_data()
    dpdx = 0.0
    for t in range(n):
        u, dpdx = nse.perform_time_step(u, dpdx, t)
        if t == 0:
            assert rel(u.cpu().numpy(), d["u1"]) < TOL
    assert rel(u.cpu().numpy(), d["un"]) < TOL
    # the same run through solve_scan (one step per launch sequence, base updated in between)
    nse2 = NavierStokesVelVortPerturbationInstationary(_vf(d), Re=float(d["re"]), dt=dt, end_time=n * dt,
                                                       kappa=float(d["kappa"]), accelerate=True,
                                                       n_max=int(d["n_max"]))
    nse2.solve_scan()
    assert rel(nse2.get_latest_field("velocity_hat").get_data().cpu().numpy(), d["un"]) < TOL


def test_coupling_off_and_linearise_switch_match_reference(cuda):
    d = golden("coupling_off_9x33x9")
    n, dt = int(d["n_steps"]), float(d["dt"])
    nse = NavierStokesVelVortPerturbation(_vf(d), Re=float(d["re"]), dt=dt, end_time=n * dt, coupling_term=False,
                                          linearise_switch=float(d["linearise_switch"]))
    nse.solve_scan()
    assert rel(nse.get_latest_field("velocity_hat").get_data().cpu().numpy(), d["un"]) < TOL
    u = nse.get_initial_field("velocity_hat").get_data()
    u1, _ = nse.perform_time_step(u, 0.0, 0)
    assert rel(u1.cpu().numpy(), d["u1"]) < TOL
