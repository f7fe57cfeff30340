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


def _problem(d, mode="gain", end_scale=1, u0_key="u0"):
    shape, (lx, lz) = tuple(int(x) for x in d["shape"]), d["lengths"]
    n, dt = int(d["n_steps"]), float(d["dt"])
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz), aliasing=3 / 2)
    u0 = VectorField.FromData(FourierField, dom, torch.as_tensor(d[u0_key], device="cuda"), name="velocity_hat")
    nse = NavierStokesVelVortPerturbation(u0, Re=float(d["re"]), dt=dt, end_time=end_scale * n * dt, linearise=True)
    return NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse, optimisation_mode=mode)


@pytest.mark.parametrize("mode", ["gain_3d", "gain_no_00", "dissipation"])
def test_dual_objectives_match_reference(cuda, mode):
    """gain_3d (u(T) without its kx = 0 part), gain_no_00 (without its (0, 0)
    mode) and dissipation (the time average of the squared velocity gradients,
    whose dual starts from zero and is driven by a source from the forward
    history in every step): objective value and dual gradient against the
    reference's dual solver (navier_stokes_perturbation_dual.py:388-400,
    904-990, 1065-1104; the source enters at navier_stokes.py:1461-1491,
    1697-1703)."""
    d = golden("dual_modes_9x33x9")
    # the dissipation case starts with a mean-flow perturbation: the objective
    # only sees the (0, 0) mode
    dual = _problem(d, mode, u0_key="dissipation_u0" if mode == "dissipation" else "u0")
    value = dual.get_objective_fun()
    assert abs(value / float(d[mode + "_value"]) - 1) < 1e-10
    grad = dual.get_grad().cpu().numpy()
    assert rel(grad, d[mode + "_grad"]) < 1e-10


def test_cg_line_search_matches_reference(cuda):
    """ConjugateGradientDescentSolver with use_linesearch: values, step sizes
    and final guess of 3 iterations against the reference solver
    (gradient_descent_solver.py:522-708)."""
    d = golden("solvers_5x33x5")
    solver = ConjugateGradientDescentSolver(_problem(d), max_iterations=3, step_size=1e-2, use_linesearch=True)
    solver.initialise()
    values, steps = [], []
    for _ in range(3):
        solver.update()
        values.append(solver.value)
        steps.append(solver.step_size)
        solver.i += 1
    assert np.abs(np.array(values) / d["ls_values"] - 1).max() < 1e-9
    np.testing.assert_allclose(steps, d["ls_steps"], rtol=1e-12)
    assert rel(solver.current_guess.get_data().cpu().numpy(), d["ls_final"]) < 1e-8


def test_steepest_adaptive_descent_matches_reference(cuda):
    """SteepestAdaptiveDescentSolver (gradient_descent_solver.py:340-488):
    initialisation and 2 updates against the reference solver (whose
    CFL-chosen dt leaves the step in use unchanged)."""
    from jax_spectral_dns.gradient_descent_solver import SteepestAdaptiveDescentSolver

    d = golden("solvers_5x33x5")
    st = SteepestAdaptiveDescentSolver(_problem(d, end_scale=10), max_iterations=3, step_size=1e-2)
    st.initialise()
    values, steps, dts = [st.value], [st.step_size], [st.dual_problem.forward_equation.get_dt()]
    for _ in range(2):
        st.update()
        values.append(st.value)
        steps.append(st.step_size)
        dts.append(st.dual_problem.forward_equation.get_dt())
        st.i += 1
    np.testing.assert_allclose(dts, d["sd_dts"], rtol=1e-13)
    assert st.cfl_dt > 0
    np.testing.assert_allclose(steps, d["sd_steps"], rtol=1e-12)
    assert np.abs(np.array(values) / d["sd_values"] - 1).max() < 1e-9
    assert rel(st.current_guess.get_data().cpu().numpy(), d["sd_final"]) < 1e-8
