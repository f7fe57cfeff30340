"""Dual-driven gain ascent (drop-in for the reference's
jax_spectral_dns/gradient_descent_solver.py, ConjugateGradientDescentSolver).

Each iteration (gradient_descent_solver.py:710-860, default path without line
search): forward run for the objective (gain), dual run for the projected
conjugate gradient (navier_stokes_perturbation_dual.py:1122-1201), step of
size `step_size` along it, renormalisation to the initial energy E0
(:307-316), step-size adaptation (x1.5 after a gain increase up to
max_step_size, /2 after a decrease down to min_step_size) and the
Polak-Ribiere coefficient beta = g.(g - g_old) / g_old.g_old of the steepest
gradients (unconjugated dot product of the flattened complex arrays, reset to
0 when its real part is negative or after a failed step, :840-851). The first
iteration limits the step to max_step_size_initial_factor times the largest
admissible projected step (:502-530).
"""
from __future__ import annotations

import math
from typing import Any, Optional

import torch

from .equation import print_verb
from .field import FourierField, VectorField
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
        self.use_linesearch = params.get("use_linesearch", False)
        if self.use_linesearch:
            raise NotImplementedError("the line-search variant is not supported")
        self.current_guess: VectorField = nse.get_initial_field("velocity_hat")
        self.history = []

    @property
    def e_0(self) -> float:
        return self._e_0

    def increase_step_size(self, tau: float = 1.5) -> None:
        self.step_size = min(self.max_step_size, self.step_size * tau)

    def decrease_step_size(self, tau: float = 2.0) -> None:
        self.step_size = max(self.step_size / tau, self.min_step_size)

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

    def update(self) -> None:
        dual = self.dual_problem
        dual.forward_equation.set_initial_field("velocity_hat", self.current_guess)
        dual.update_with_nse()
        gain = dual.get_objective_fun()
        gain_change = gain - self.value if self.value is not None else None
        print_verb("iteration", self.i + 1, dual.get_objective_fun_name(), gain, verbosity_level=1)
        if self.old_grad is not None:
            self.grad, _ = dual.get_projected_cg_grad(self.step_size, self.beta, self.old_grad)
            self.steepest_grad, _ = dual.get_projected_grad(self.step_size)
        else:
            self.grad, _ = dual.get_projected_grad(self.step_size,
                                                   step_size_factor=self.max_step_size_initial_factor)
            self.steepest_grad = self.grad
            self.step_size = min(self.step_size, self.get_max_step_size_ls() * self.max_step_size_initial_factor)
        guess = VectorField.FromData(FourierField, dual.get_physical_domain(),
                                     self.current_guess.get_data() + self.step_size * self.grad,
                                     name="velocity_hat")
        self.current_guess = self.normalize_field(guess)
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
