"""Gain G = E(T)/E(0) as a differentiable torch function.

The reference obtains the gradient of the transient-growth gain either with
jax.value_and_grad through the forward solve (optimiser.py:120) or with its
dual solver (navier_stokes_perturbation_dual.py:850-1120): forward run, dual run
backward from -u(T) with Re and dt negated (dual step t frozen at the forward
state u(T - t)), gradient (u0 - v0) / E0 in the energy inner product. This
module provides both behind ``torch.autograd.Function``:

* ``gradient="discrete"`` (the default for the linearised equations): the
  exact derivative of the computed gain, like jax.grad of the forward solve.
  The linearised step is a fixed linear map S, so dG/du0 =
  (S^T)^N grad E(u_N) / E0 - G grad E(u0) / E0, with S^T applied by the
  hand-written transpose of the step (jsd_step_adjoint) and grad E by
  jsd_energy_grad; no forward states are kept, and the cost is one forward and
  one adjoint pass.
* ``gradient="dual"`` (the nonlinear equations): the reference's continuous
  dual. Forward: N = int(T/dt) native forward steps, keeping the state every
  K steps (checkpoints) instead of the whole trajectory; backward: for each
  K-step segment, last first, recompute the segment's K + 1 forward states
  from its checkpoint (only the nonlinear dual needs them), register them with
  the dual plan and take K dual steps. Memory is N/K + K + 1 states instead of
  N + 1; the cost is one forward pass, one recompute pass and one dual pass
  (about 3 forward costs). With K >= N the forward pass itself records the
  N + 1 states (there is one segment and nothing to recompute): N + 1 states
  of memory, one forward and one dual pass. The continuous dual approximates
  the derivative of the discrete gain (to O(dt), and less well where the
  dealiasing truncation matters).

Gradients. With the dual field v0 (the dual run started from -u(T)),
dE(T) = <-v0, du> and dE(0) = <u0, du> in the energy inner product
<a, b> = (1/V) int a . b, so the full derivative of G is
dG = <(-v0 - G u0) / E0, du>. The reference's ``get_grad`` returns
(u0 - v0) / E0, which equals it along directions orthogonal to u0 (the
energy sphere its optimisers move on); ``dual_gradient`` returns that
reference quantity. The autograd gradient is the Euclidean one for the real
and imaginary parts of the spectral coefficients (torch's convention for a
real loss of a complex input), so that sum Re(conj(grad) * du) = dG; for the
dual it is the energy-metric gradient scaled by 2 * (c^2/4) * w_y per
coefficient, exact for Hermitian du.
"""
from __future__ import annotations

import math
from typing import Optional

import torch

from . import _native
from ._ops import operator_tables
from ._plan import GraphedSteps, StepPlan, to_device_layout, to_reference_layout
from .seeds import cheb_points


class GainProblem:
    """Forward and dual plans for a perturbation problem about U = u_max (1 - y^2)."""

    def __init__(self, modes, phys, lx, lz, re, dt, end_time, linearise, u_max=1.0, checkpoint_every=10,
                 precision="fp64", device="cuda", use_graphs=True, gradient: Optional[str] = None):
        self.modes, self.phys = tuple(modes), tuple(phys)
        self.lx, self.lz = float(lx), float(lz)
        self.re_tau = float(re) / u_max
        self.dt = float(dt)
        self.n_steps = max(0, int(end_time / dt))
        self.linearise = bool(linearise)
        if gradient is None:
            gradient = "discrete" if self.linearise else "dual"
        if gradient not in ("discrete", "dual"):
            raise ValueError("gradient must be 'discrete' or 'dual'")
        if gradient == "discrete" and not self.linearise:
            raise ValueError("the discrete adjoint covers the linearised equations; use gradient='dual'")
        self.gradient = gradient
        self.K = max(1, min(int(checkpoint_every), max(1, self.n_steps)))
        self.full_trajectory = self.K >= self.n_steps  # one segment: record it in the forward pass
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
        # fixed working buffers so segments can replay captured CUDA graphs
        self.use_graphs = use_graphs
        shape = (3, ny, self.modes[0], self.modes[2])
        self.w_fwd = torch.zeros(shape, dtype=torch.complex128, device=device)
        self.w_dual = torch.zeros(shape, dtype=torch.complex128, device=device)
        self.w_dp = torch.zeros(1, dtype=torch.float64, device=device)
        self.w_ddp = torch.zeros(1, dtype=torch.float64, device=device)
        self.w_traj = torch.zeros((self.K + 1,) + shape, dtype=torch.complex128, device=device)
        self.w_adj = torch.zeros(shape, dtype=torch.complex128, device=device)
        self.w_traj2 = None  # second segment buffer of the pipelined recompute (allocated on first use)
        self._side = None
        self._graphs = {}
        self._traj_owner = None  # checkpoint list of the forward pass whose trajectory w_traj holds

    def _run(self, key, make):
        """Replay the captured graph for `key` (capture on first use)."""
        if not self.use_graphs:
            make(None)
            return
        g = self._graphs.get(key)
        if g is None:
            g = self._graphs[key] = make(True)
        g.replay()

    def _fwd_steps(self, n: int) -> None:
        def make(capture):
            if capture:
                return GraphedSteps(self.fwd, self.w_fwd, self.w_dp, 0, n)
            self.fwd.step(self.w_fwd, self.w_dp, 0, n)
        self._run(("fwd", n), make)

    def _traj_buf(self, b: int) -> torch.Tensor:
        if b == 0:
            return self.w_traj
        if self.w_traj2 is None:
            self.w_traj2 = torch.zeros_like(self.w_traj)
        return self.w_traj2

    def _fwd_traj(self, n: int, b: int = 0) -> None:
        traj_buf = self._traj_buf(b)

        def make(capture):
            if capture:
                return GraphedSteps(self.fwd, self.w_fwd, self.w_dp, 0, n, trajectory=traj_buf)
            traj = self.fwd.step_trajectory(self.w_fwd, self.w_dp, 0, n)
            traj_buf[: n + 1].copy_(traj)
        self._run(("traj", n, b), make)

    def _dual_steps(self, n: int, b: int = 0) -> None:
        traj_buf = self._traj_buf(b)

        def make(capture):
            if not self.linearise:
                self.dual.set_history(traj_buf[: n + 1])
            if capture:
                return GraphedSteps(self.dual, self.w_dual, self.w_ddp, 0, n)
            self.dual.step(self.w_dual, self.w_ddp, 0, n)
        self._run(("dual", n, b), make)

    def _adj_steps(self, n: int) -> None:
        """w_adj <- (S^T)^n w_adj (discrete adjoint of n linearised steps)."""
        if not self.use_graphs:
            self.fwd.step_adjoint(self.w_adj, n)
            return
        g = self._graphs.get(("adj", n))
        if g is None:
            probe = self.w_adj.clone()
            self.fwd.step_adjoint(probe, n)  # loads every kernel before the capture
            torch.cuda.synchronize(self.w_adj.device)
            g = torch.cuda.CUDAGraph()
            stream = torch.cuda.Stream(device=self.w_adj.device)
            stream.wait_stream(torch.cuda.current_stream(self.w_adj.device))
            with torch.cuda.stream(stream):
                with torch.cuda.graph(g, stream=stream):
                    self.fwd.step_adjoint(self.w_adj, n)
            torch.cuda.current_stream(self.w_adj.device).wait_stream(stream)
            self._graphs[("adj", n)] = g
        g.replay()

    def forward_only(self, u0_dev: torch.Tensor) -> torch.Tensor:
        """u(T) from u0 (no checkpoints: the linearised adjoint needs none)."""
        self.w_fwd.copy_(u0_dev)
        self.w_dp.zero_()
        t = 0
        while t < self.n_steps:
            n = min(self.K, self.n_steps - t)
            self._fwd_steps(n)
            t += n
        self.fwd.check_device_errors()
        return self.w_fwd.clone()

    def discrete_gradient(self, u0_dev: torch.Tensor, uT: Optional[torch.Tensor] = None):
        """(gain, dG/du0) with the exact transpose of the linearised step:
        dG/du0 = (S^T)^N grad E(u_N) / E0 - G grad E(u0) / E0, device layout,
        Euclidean in the real and imaginary parts."""
        if uT is None:
            uT = self.forward_only(u0_dev)
        e0 = self.energy(u0_dev)
        gain = self.energy(uT) / e0
        self.w_adj.copy_(self.fwd.energy_grad(uT) / e0)
        t = 0
        while t < self.n_steps:
            n = min(self.K, self.n_steps - t)
            self._adj_steps(n)
            t += n
        self.fwd.check_device_errors()
        grad = self.w_adj - (gain / e0) * self.fwd.energy_grad(u0_dev)
        return gain, grad

    # ---- pieces ----------------------------------------------------------
    def energy(self, state: torch.Tensor) -> torch.Tensor:
        return self.fwd.energy(state)

    def forward_checkpoints(self, u0_dev: torch.Tensor):
        """Run all steps; return the final state and the states at steps 0, K, 2K, ...
        (with one segment and a nonlinear dual, the whole trajectory is kept in
        the working buffer instead)."""
        self.w_fwd.copy_(u0_dev)
        self.w_dp.zero_()
        cps = [u0_dev.clone()]
        if self.full_trajectory and not self.linearise and self.n_steps > 0:
            self._fwd_traj(self.n_steps)
            self._traj_owner = cps  # the recorded trajectory belongs to this forward pass
            self.fwd.check_device_errors()
            return self.w_fwd.clone(), cps
        self._traj_owner = None
        t = 0
        while t < self.n_steps:
            n = min(self.K, self.n_steps - t)
            self._fwd_steps(n)
            t += n
            if t < self.n_steps:
                cps.append(self.w_fwd.clone())
        self.fwd.check_device_errors()
        return self.w_fwd.clone(), cps

    def backward_dual(self, uT: torch.Tensor, cps) -> torch.Tensor:
        """Dual run from -u(T) to t = 0, recomputing each segment's forward
        states from its checkpoint when the dual needs them. The recompute of
        the next segment (on a second stream, into the other of two segment
        buffers) overlaps the dual run over the current one; events order each
        dual run after its segment's recompute and each recompute after the
        dual run that last read its buffer."""
        self.w_dual.copy_(-uT)
        self.w_ddp.zero_()
        bounds = list(range(0, self.n_steps, self.K)) + [self.n_steps]
        segs = list(range(len(bounds) - 2, -1, -1))  # last segment first
        recorded = self._traj_owner is cps and len(bounds) == 2
        if self.linearise or recorded:
            # no recompute: the linear dual needs no forward states, and a
            # single segment recorded by this forward pass is already in w_traj
            for seg in segs:
                self._dual_steps(bounds[seg + 1] - bounds[seg])
        else:
            main = torch.cuda.current_stream(self.w_dual.device)
            if self._side is None:
                self._side = torch.cuda.Stream(device=self.w_dual.device)
            side = self._side
            ready = [torch.cuda.Event(), torch.cuda.Event()]
            free = [torch.cuda.Event(), torch.cuda.Event()]
            side.wait_stream(main)

            def recompute(i):
                seg, b = segs[i], i % 2
                with torch.cuda.stream(side):
                    if i >= 2:
                        side.wait_event(free[b])  # the dual run two segments back read this buffer
                    self.w_fwd.copy_(cps[seg])
                    self.w_dp.zero_()
                    self._fwd_traj(bounds[seg + 1] - bounds[seg], b)
                    ready[b].record(side)

            recompute(0)
            for i, seg in enumerate(segs):
                if i + 1 < len(segs):
                    recompute(i + 1)
                b = i % 2
                main.wait_event(ready[b])
                # dual step t of this segment uses the segment state n - t
                self._dual_steps(bounds[seg + 1] - bounds[seg], b)
                free[b].record(main)
            main.wait_stream(side)
            self._traj_owner = None  # the segment buffers now hold recomputed segments
        self.fwd.check_device_errors()
        self.dual.check_device_errors()
        return self.w_dual.clone()

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
        if problem.gradient == "discrete":
            uT, cps = problem.forward_only(u0_dev), None
        else:
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
        if problem.gradient == "discrete":
            _, g_euc = problem.discrete_gradient(u0_dev, uT)
            return to_reference_layout(g_euc).to(ctx.in_device) * grad_out.to(ctx.in_device), None
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
