"""Gain G = E(T)/E(0) as a differentiable torch function, backward by the dual step.

The reference obtains the gradient of the transient-growth gain either with
jax.value_and_grad through the forward solve (optimiser.py:120) or with its
dual solver (navier_stokes_perturbation_dual.py:850-1120): forward run, dual run
backward from -u(T) with Re and dt negated (dual step t frozen at the forward
state u(T - t)), gradient (u0 - v0) / E0 in the energy inner product. This
module puts the dual-solver gradient behind ``torch.autograd.Function``:

* forward: N = int(T/dt) native forward steps, keeping the state every K steps
  (checkpoints) instead of the whole trajectory;
* backward: for each K-step segment, last first, recompute the segment's
  K + 1 forward states from its checkpoint (only the nonlinear dual needs
  them), register them with the dual plan and take K dual steps.

Memory is N/K + K + 1 states instead of N + 1; the cost is one forward pass,
one recompute pass and one dual pass (about 3 forward costs).

Gradients. With the dual field v0 (the dual run started from -u(T)),
dE(T) = <-v0, du> and dE(0) = <u0, du> in the energy inner product
<a, b> = (1/V) int a . b, so the full derivative of G is
dG = <(-v0 - G u0) / E0, du>. The reference's ``get_grad`` returns
(u0 - v0) / E0, which equals it along directions orthogonal to u0 (the
energy sphere its optimisers move on); ``dual_gradient`` returns that
reference quantity, the autograd backward returns the full derivative. The
autograd gradient is the Euclidean one for the real and imaginary parts of
the spectral coefficients (torch's convention for a real loss of a complex
input): the energy-metric gradient scaled by 2 * (c^2/4) * w_y per
coefficient, so that sum Re(conj(grad) * du) = dG for Hermitian du.
"""
from __future__ import annotations

import math
from typing import Optional

import torch

from . import _native
from ._ops import operator_tables
from ._plan import StepPlan, to_device_layout, to_reference_layout
from .seeds import cheb_points


class GainProblem:
    """Forward and dual plans for a perturbation problem about U = u_max (1 - y^2)."""

    def __init__(self, modes, phys, lx, lz, re, dt, end_time, linearise, u_max=1.0, checkpoint_every=10,
                 precision="fp64", device="cuda"):
        self.modes, self.phys = tuple(modes), tuple(phys)
        self.lx, self.lz = float(lx), float(lz)
        self.re_tau = float(re) / u_max
        self.dt = float(dt)
        self.n_steps = max(0, int(end_time / dt))
        self.linearise = bool(linearise)
        self.K = max(1, int(checkpoint_every))
        ny = self.modes[1]
        base = u_max * (1 - cheb_points(ny) ** 2)
        self.fwd = StepPlan(modes, phys, lx, lz, _native.JSD_KIND_PERTURBATION, self.re_tau, self.dt,
                            linearise=linearise, base_u=base, precision=precision, device=device)
        self.dual = StepPlan(modes, phys, lx, lz, _native.JSD_KIND_DUAL, self.re_tau, self.dt,
                             dt_explicit=-self.dt, linearise=linearise, base_u=base, precision=precision,
                             device=device)
        s = (self.lx / (2 * math.pi)) * (self.lz / (2 * math.pi))
        c = s / math.sqrt(self.phys[0] * self.phys[-1])
        w = torch.as_tensor(operator_tables(ny).y_weights, dtype=torch.float64, device=device)
        # Euclidean gradient = energy gradient * 2 * (c^2 / 4) * w_y (device layout (3, Ny, Mx, Mz))
        self.metric = (0.5 * c * c * w).view(1, ny, 1, 1)

    # ---- pieces ----------------------------------------------------------
    def energy(self, state: torch.Tensor) -> torch.Tensor:
        return self.fwd.energy(state)

    def forward_checkpoints(self, u0_dev: torch.Tensor):
        """Run all steps; return the final state and the states at steps 0, K, 2K, ..."""
        st = u0_dev.clone()
        dp = torch.zeros(1, dtype=torch.float64, device=st.device)
        cps = [st.clone()]
        t = 0
        while t < self.n_steps:
            n = min(self.K, self.n_steps - t)
            self.fwd.step(st, dp, t, n)
            t += n
            if t < self.n_steps:
                cps.append(st.clone())
        return st, cps

    def backward_dual(self, uT: torch.Tensor, cps) -> torch.Tensor:
        """Dual run from -u(T) to t = 0, recomputing each segment's forward
        states from its checkpoint when the dual needs them."""
        v = (-uT).contiguous()
        dp = torch.zeros(1, dtype=torch.float64, device=v.device)
        bounds = list(range(0, self.n_steps, self.K)) + [self.n_steps]
        for seg in range(len(bounds) - 2, -1, -1):
            s0, s1 = bounds[seg], bounds[seg + 1]
            n = s1 - s0
            if not self.linearise:
                traj = torch.empty((n + 1,) + tuple(v.shape), dtype=v.dtype, device=v.device)
                traj[0].copy_(cps[seg])
                st = cps[seg].clone()
                fdp = torch.zeros(1, dtype=torch.float64, device=v.device)
                for k in range(n):
                    self.fwd.step(st, fdp, s0 + k, 1)
                    traj[k + 1].copy_(st)
                self.dual.set_history(traj)
            # dual step t of this segment uses the segment state n - t
            self.dual.step(v, dp, 0, n)
            if not self.linearise:
                self.dual.set_history(None)
        return v

    def gain_and_dual(self, u0_dev: torch.Tensor):
        uT, cps = self.forward_checkpoints(u0_dev)
        e0 = self.energy(u0_dev)
        gain = self.energy(uT) / e0
        v0 = self.backward_dual(uT, cps)
        return gain, (u0_dev - v0) / e0, uT


class _Gain(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, problem: GainProblem):
        u0_dev = to_device_layout(u0.detach(), device=problem.fwd.device)
        uT, cps = problem.forward_checkpoints(u0_dev)
        e0 = problem.energy(u0_dev)
        gain = problem.energy(uT) / e0
        ctx.problem = problem
        ctx.saved = (u0_dev, uT, cps, e0)
        ctx.in_device = u0.device
        return gain.reshape(()).to(u0.device)

    @staticmethod
    def backward(ctx, grad_out):
        problem = ctx.problem
        u0_dev, uT, cps, e0 = ctx.saved
        v0 = problem.backward_dual(uT, cps)
        G = problem.energy(uT) / e0
        g_energy = (-v0 - G * u0_dev) / e0
        g_euc = g_energy * problem.metric
        return to_reference_layout(g_euc).to(ctx.in_device) * grad_out.to(ctx.in_device), None


def gain(u0: torch.Tensor, problem: GainProblem) -> torch.Tensor:
    """Differentiable gain E(T)/E(0) of a (3, Mx, Ny, Mz) complex128 spectral field."""
    return _Gain.apply(u0, problem)


def dual_gradient(u0: torch.Tensor, problem: GainProblem):
    """(gain, energy-metric gradient (u0 - v0)/E0 in the reference layout) --
    the quantity NavierStokesVelVortPerturbationDual.get_grad returns."""
    u0_dev = to_device_layout(u0, device=problem.fwd.device)
    g, grad, _ = problem.gain_and_dual(u0_dev)
    return float(g.item()), to_reference_layout(grad)
