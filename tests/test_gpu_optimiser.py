"""Dual-driven conjugate-gradient gain ascent against the reference's
ConjugateGradientDescentSolver (golden: 5 iterations, pseudo-2D 5x33x5)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.field import FourierField, VectorField
from jax_spectral_dns.gradient_descent_solver import ConjugateGradientDescentSolver
from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation
from jax_spectral_dns.navier_stokes_perturbation_dual import NavierStokesVelVortPerturbationDual

pytestmark = pytest.mark.gpu


def test_cg_gain_ascent_matches_reference(cuda):
    d = golden("cg_opt_5x33x5")
    shape, (lx, lz) = tuple(d["shape"]), d["lengths"]
    n, dt = int(d["n_steps"]), float(d["dt"])
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz), aliasing=3 / 2)
    u0 = VectorField.FromData(FourierField, dom, torch.as_tensor(d["u0"], device="cuda"), name="velocity_hat")
    nse = NavierStokesVelVortPerturbation(u0, Re=float(d["re"]), dt=dt, end_time=n * dt, linearise=True)
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
    solver = ConjugateGradientDescentSolver(dual, max_iterations=5, step_size=1e-2)
    solver.initialise()
    while not solver.is_done(solver.i):
        solver.update()
        solver.i += 1
    gains = np.array(solver.history)
    assert gains.shape == d["gains"].shape
    assert np.abs(gains / d["gains"] - 1).max() < 1e-9
    assert rel(solver.current_guess.get_data().cpu().numpy(), d["final_guess"]) < 1e-8
