"""Dual-driven gain ascent (drop-in for the reference's
jax_spectral_dns/gradient_descent_solver.py: ConjugateGradientDescentSolver,
SteepestAdaptiveDescentSolver).

Conjugate gradients, each iteration (gradient_descent_solver.py:710-860):
forward run for the objective, dual run for the projected conjugate gradient
(navier_stokes_perturbation_dual.py:1122-1201), step of size `step_size`
along it, renormalisation to the initial energy E0 (:307-316), step-size
adaptation (x1.5 after a gain increase up to max_step_size, /2 after a
decrease down to min_step_size) and the Polak-Ribiere coefficient
beta = g.(g - g_old) / g_old.g_old of the steepest gradients (unconjugated
dot product of the flattened complex arrays, reset to 0 when its real part
is negative or after a failed step, :840-851). The first iteration limits the
step to max_step_size_initial_factor times the largest admissible projected
step (:502-530). With use_linesearch the step size comes from the line
search of :522-708 (Armijo constant 0, so a step is accepted when the
objective grows: grown by 1.5 while it keeps growing every
linesearch_increase_interval iterations, halved while it falls), and beta
stays 0 as in the reference (no value change is recorded on that path).

Steepest adaptive descent (:340-488): a step along the projected gradient;
if the objective fell, the step size is divided by 5 and the step is retried
from the previous gradient (at most max_number_of_sub_iterations times),
else the step size grows by 1.5. After every iteration the reference chooses
a dt from the CFL number of the final velocity plus base flow
(Equation.find_suitable_dt) and hands it to update_dt, which leaves get_dt()
unchanged, so the trial problems keep the original step; that dt is kept in
`cfl_dt`.
As in the reference, the forward problem of every trial step is a new
NavierStokesVelVortPerturbation with the default (nonlinear) equations, and
after an update the old and new values coincide, so `optimise` stops after
one iteration through the relative-change test.
"""
from __future__ import annotations

import math
from typing import Any, Optional

import torch

from .equation import Equation, print_verb
from .field import FourierField, VectorField
from .navier_stokes_perturbation import NavierStokesVelVortPerturbation
from .navier_stokes_perturbation_dual import NavierStokesVelVortPerturbationDual


class GradientDescentSolver:
    def __init__(self, dual_problem: NavierStokesVelVortPerturbationDual, **params: Any):
        self.dual_problem = dual_problem
        nse = dual_problem.forward_equation
        self._e_0 = nse.energy_of(nse.get_initial_field("velocity_hat").get_data())
        self.done = False
        self.post_process_fn = params.get("post_process_function", None)
        self.value: Optional[float] = None
        self.old_value: Optional[float] = None
        self.i = params.get("start_iteration", 0)
        if self.i < 0:
            raise NotImplementedError("resuming from saved fields is not supported")
        self.max_step_size = params.get("max_step_size", 1e-1)
        self.min_step_size = params.get("min_step_size", 1e-4)
        self.step_size = params.get("step_size", 1e-2)
        self.max_step_size_initial_factor = params.get("max_step_size_initial_factor", 1.25e-1)
        self.number_of_steps = params.get("max_iterations", 20)
        self.value_change_threshold = params.get("value_change_threshold", 1e-8)
        self.max_number_of_sub_iterations = params.get("max_number_of_sub_iterations", 10)
        self.use_linesearch = params.get("use_linesearch", False)
        self.linesearch_increase_interval = params.get("linesearch_increase_interval", 3)
        self.current_guess: VectorField = nse.get_initial_field("velocity_hat")
        self.history = []

    @property
    def e_0(self) -> float:
        return self._e_0

    def increase_step_size(self, tau: float = 1.5) -> None:
        self.step_size = min(self.max_step_size, self.step_size * tau)

    def decrease_step_size(self, tau: float = 5.0) -> None:
        self.step_size /= tau

    def normalize_current_guess(self) -> None:
        self.current_guess = self.normalize_field(self.current_guess)

    def is_done(self, i: int) -> bool:
        return (i >= self.number_of_steps) or (
            self.value is not None and self.old_value is not None
            and abs((self.value - self.old_value) / self.value) < self.value_change_threshold)

    def normalize_field(self, v0_hat: VectorField) -> VectorField:
        """Physical round trip and rescaling to the initial energy."""
        v0 = v0_hat.no_hat()
        en = v0.energy()
        v0 = v0 * (math.sqrt(self.e_0) / math.sqrt(en))
        out = v0.hat()
        out.set_name("velocity_hat")
        return out

    def optimise(self, **params: Any) -> None:
        self.initialise()
        while not self.is_done(self.i):
            self.update()
            self.i += 1
            assert self.value is not None and math.isfinite(self.value), "calculation failure detected."
        self.perform_final_run()

    def perform_final_run(self) -> float:
        dual = self.dual_problem
        dual.forward_equation.set_initial_field("velocity_hat", self.current_guess)
        dual.update_with_nse()
        value = dual.get_objective_fun()
        print_verb("final", dual.get_objective_fun_name() + ":", value)
        self.old_value, self.value = self.value, value
        return value


class SteepestAdaptiveDescentSolver(GradientDescentSolver):
    def _suitable_dt(self, dual) -> float:
        """dt from the CFL number of u(T) + base flow (gradient_descent_solver.py:355-368)."""
        nse = dual.forward_equation
        vT = nse.get_latest_field("velocity_hat").no_hat() + nse.get_initial_field("velocity_base_hat").no_hat()
        return Equation.find_suitable_dt(nse.get_physical_domain(), nse.max_cfl,
                                         tuple(vT[i].max() for i in range(3)), nse.end_time)

    def _retime(self, dual, dt: float) -> None:
        """The reference calls update_dt(dt) here (gradient_descent_solver.py:
        369-370, 474-475), which rebuilds the implicit matrices for dt while
        get_dt() keeps the old step (navier_stokes.py:810-873); every later
        trial problem is built with get_dt() and never reads those matrices,
        so the step in use stays the same. The CFL step is kept for inspection."""
        self.cfl_dt = dt

    def initialise(self, prepare_for_iterations: bool = True) -> None:
        self.current_guess.set_name("velocity_hat")
        nse = self.dual_problem.forward_equation
        self.dual_problem = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
        if prepare_for_iterations:
            self.value = self.dual_problem.get_objective_fun()
            dt = self._suitable_dt(self.dual_problem)
            self.grad, _ = self.dual_problem.get_projected_grad(self.step_size)
            self.old_value = self.value
            self.old_nse_dual = self.dual_problem
            self._retime(self.dual_problem, dt)
            print_verb(self.dual_problem.get_objective_fun_name(), self.value)

    def update(self) -> None:
        v0_hat = self.current_guess
        domain = v0_hat.get_physical_domain()
        j = 0
        while True:
            print_verb("iteration", self.i + 1, "step size:", self.step_size, verbosity_level=2)
            v0_new = self.normalize_field(VectorField.FromData(FourierField, domain,
                                                               v0_hat.get_data() + self.step_size * self.grad,
                                                               name="velocity_hat"))
            v0_new.set_name("velocity_hat")
            nse_ = self.dual_problem.forward_equation
            nse = NavierStokesVelVortPerturbation(v0_new, Re=nse_.get_Re_tau() * nse_.get_u_max_over_u_tau(),
                                                  dt=nse_.get_dt(), end_time=nse_.end_time,
                                                  velocity_base_hat=nse_.get_latest_field("velocity_base_hat"))
            self.dual_problem = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse)
            gain = self.dual_problem.get_objective_fun()
            print_verb(self.dual_problem.get_objective_fun_name(), gain)
            gain_change = gain - self.old_value
            if gain_change > 0.0:
                done = True
                self.increase_step_size()
                self.grad, _ = self.dual_problem.get_projected_grad(self.step_size)
            else:
                done = False
                self.decrease_step_size()
                self.grad, _ = self.old_nse_dual.get_projected_grad(self.step_size)
                print_verb("gain decrease/stagnation detected, repeating iteration with smaller step size.")
            j += 1
            if done or j > self.max_number_of_sub_iterations:
                break
        self._retime(self.dual_problem, self._suitable_dt(self.dual_problem))
        self.current_guess = v0_new
        self.normalize_current_guess()
        self.old_nse_dual = self.dual_problem
        self.value = gain
        self.old_value = self.value
        self.history.append(gain)


class ConjugateGradientDescentSolver(GradientDescentSolver):
    def initialise(self, prepare_for_iterations: bool = True) -> None:
        self.beta = 0.0
        self.current_guess.set_name("velocity_hat")
        self.dual_problem.update_with_nse()
        self.value = None
        self.old_value = None
        self.old_grad: Optional[torch.Tensor] = None
        self.old_steepest_grad: Optional[torch.Tensor] = None

    def get_max_step_size_ls(self) -> float:
        dual = self.dual_problem
        nse = dual.forward_equation
        u0 = dual.velocity_u_hat_0.get_data()
        v0 = dual.get_latest_field("velocity_hat").get_data()
        if self.old_grad is not None:
            v0 = v0 - self.beta * self.old_grad
        e_adj = nse.energy_of(v0)
        c0 = nse.energy_of(u0 + v0) - nse.energy_of(u0) - e_adj
        return (e_adj / self.e_0 - c0 ** 2 / (4 * self.e_0 ** 2)) ** (-1 / 2)

    def increase_step_size(self, tau: float = 1.5) -> None:
        if self.use_linesearch:
            self.step_size = min(self.get_max_step_size_ls(), self.step_size * tau)
        else:
            self.step_size = min(self.max_step_size, self.step_size * tau)

    def decrease_step_size(self, tau: float = 2.0) -> None:
        self.step_size = max(self.step_size / tau, self.min_step_size)

    def _direction(self, step_size, u_hat_0=None, v_hat_0=None):
        dual = self.dual_problem
        if self.old_grad is not None:
            return dual.get_projected_cg_grad(step_size, self.beta, self.old_grad, u_hat_0, v_hat_0)[0]
        return dual.get_projected_grad(step_size, u_hat_0, v_hat_0)[0]

    def _evaluate(self, guess: VectorField) -> float:
        dual = self.dual_problem
        dual.forward_equation.set_initial_field("velocity_hat", guess)
        dual.update_with_nse()
        return dual.get_objective_fun()

    def get_step_size_ls(self, old_value: float):
        """Line search (gradient_descent_solver.py:522-708) with Armijo
        constant c = 0: returns (step size, objective) and leaves the accepted
        guess in current_guess and as the forward problem's initial field."""
        dual = self.dual_problem
        step_size = self.step_size
        u_hat_0 = dual.velocity_u_hat_0
        v_hat_0 = dual.get_latest_field("velocity_hat")
        domain = dual.get_physical_domain()

        def guess_for(step):
            self.grad = self._direction(step, u_hat_0, v_hat_0)
            return self.normalize_field(VectorField.FromData(FourierField, domain,
                                                             self.current_guess.get_data() + step * self.grad,
                                                             name="velocity_hat"))

        current_guess = guess_for(step_size)
        old_current_guess = current_guess
        new_value = self._evaluate(current_guess)
        new_old_value = old_value
        print_verb("gain change:", new_value - old_value, verbosity_level=2)
        if new_value - old_value > 0.0:
            if self.i % self.linesearch_increase_interval == 0:
                while new_value >= new_old_value and new_value - old_value > 0.0 and step_size < self.max_step_size:
                    step_size *= 1.5
                    old_current_guess = current_guess
                    current_guess = guess_for(step_size)
                    new_old_value = new_value
                    new_value = self._evaluate(current_guess)
                # revert the last growth
                step_size /= 1.5
                current_guess = old_current_guess
                new_value = self._evaluate(current_guess)
                self.grad = self._direction(step_size, u_hat_0, v_hat_0)
        else:
            while new_value - old_value < 0.0 and step_size > self.min_step_size:
                step_size *= 0.5
                current_guess = guess_for(step_size)
                new_value = self._evaluate(current_guess)
        self.current_guess = current_guess
        return step_size, new_value

    def update(self) -> None:
        dual = self.dual_problem
        v0 = self.current_guess.no_hat()
        cont_error = v0.div().energy() / v0.energy()
        print_verb("continuity error:", cont_error, verbosity_level=2)
        if (not self.use_linesearch) or self.value is None:
            dual.forward_equation.set_initial_field("velocity_hat", self.current_guess)
            dual.update_with_nse()
            gain = dual.get_objective_fun()
        else:
            gain = self.value
        gain_change = gain - self.value if (self.value is not None and not self.use_linesearch) else None
        print_verb("iteration", self.i + 1, dual.get_objective_fun_name(), gain, verbosity_level=1)
        if self.old_grad is not None:
            self.grad, _ = dual.get_projected_cg_grad(self.step_size, self.beta, self.old_grad)
            self.steepest_grad, _ = dual.get_projected_grad(self.step_size)
        else:
            self.grad, _ = dual.get_projected_grad(self.step_size,
                                                   step_size_factor=self.max_step_size_initial_factor)
            self.steepest_grad = self.grad
            self.step_size = min(self.step_size, self.get_max_step_size_ls() * self.max_step_size_initial_factor)
        if self.use_linesearch:
            self.step_size, gain = self.get_step_size_ls(gain)
        else:
            guess = VectorField.FromData(FourierField, dual.get_physical_domain(),
                                         self.current_guess.get_data() + self.step_size * self.grad,
                                         name="velocity_hat")
            self.current_guess = self.normalize_field(guess)
        if dual.forward_equation.constant_mass_flux:
            self.current_guess = dual.forward_equation.update_velocity_field(self.current_guess)
        if gain_change is not None:
            if gain_change > 0.0:
                self.increase_step_size()
                self.update_beta(True)
            else:
                self.decrease_step_size()
                self.update_beta(False)
        self.old_grad = self.grad
        self.old_steepest_grad = self.steepest_grad
        self.old_value = self.value
        self.value = gain
        self.history.append(gain)

    def update_beta(self, last_iteration_successful: bool) -> None:
        if last_iteration_successful and self.old_steepest_grad is not None:
            g = self.steepest_grad.flatten()
            go = self.old_steepest_grad.flatten()
            beta = complex((torch.dot(g, g - go) / torch.dot(go, go)).item())
            self.beta = 0.0 if beta.real < 0.0 else beta
        else:
            self.beta = 0.0
