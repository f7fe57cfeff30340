"""Ensembles of independent perturbation runs on one GPU.

Every run has its own native plan (grids, Reynolds numbers and horizons
differ) and its state advances in CUDA-graph-captured chunks of steps. The
chunks of different runs are replayed on a pool of streams, so the many small
problems of an ensemble overlap on the device instead of running one after
another; ``run_sequential`` replays the same graphs on one stream for the
comparison. Runs are independent: across GPUs an ensemble is split by run
(replicas, no collective).

``draw_ensemble`` draws the benchmark ensemble: {Nx = Nz} in {16, 32, 48, 64},
Ny in {49, 65, 97}, Re uniform in [2000, 6000], E0 log-uniform in
[1e-6, 1e-2], T in {5, 10, 15, 20}, dt = 0.01, seeded solenoidal fields as for
the single runs (|kx|, |kz| <= 8).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from . import _native
from ._plan import GraphedSteps, StepPlan, to_device_layout
from .seeds import cheb_points, mode_counts, seeded_velocity_hat


@dataclass
class RunSpec:
    n: int            # Nx = Nz
    ny: int
    re: float
    e0: float
    horizon: float
    dt: float = 0.01
    seed: int = 0
    lx: float = 2 * math.pi
    lz: float = math.pi
    linearise: bool = False

    @property
    def steps(self) -> int:
        return max(0, int(self.horizon / self.dt))


def draw_ensemble(n_runs: int = 256, seed: int = 0, horizon_scale: float = 1.0) -> List[RunSpec]:
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n_runs):
        n = int(rng.choice([16, 32, 48, 64]))
        ny = int(rng.choice([49, 65, 97]))
        re = float(rng.uniform(2000.0, 6000.0))
        e0 = float(10 ** rng.uniform(-6.0, -2.0))
        horizon = float(rng.choice([5.0, 10.0, 15.0, 20.0])) * horizon_scale
        out.append(RunSpec(n, ny, re, e0, horizon, seed=seed * 100000 + i))
    return out


class Ensemble:
    def __init__(self, specs: List[RunSpec], streams: int = 16, chunk: int = 50, precision: str = "fp64",
                 device: str = "cuda"):
        self.specs = specs
        self.chunk = chunk
        self.device = torch.device(device)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, streams))]
        self.plans, self.states, self.dpdx, self.graphs = [], [], [], []
        for s in specs:
            shape = (s.n, s.ny, s.n)
            modes, phys = mode_counts(shape)
            kmax = (min(8, modes[0] // 2), min(8, modes[2] // 2))
            plan = StepPlan(modes, phys, s.lx, s.lz, _native.JSD_KIND_PERTURBATION, s.re, s.dt,
                            linearise=s.linearise, base_u=1 - cheb_points(modes[1]) ** 2, precision=precision,
                            device=device)
            u0 = seeded_velocity_hat(shape, (s.lx, s.lz), kmax, s.e0, s.seed)
            self.plans.append(plan)
            self.states.append(to_device_layout(u0, device=self.device))
            self.dpdx.append(torch.zeros(1, dtype=torch.float64, device=self.device))
        self.initial = [st.clone() for st in self.states]
        for i, plan in enumerate(self.plans):
            full = GraphedSteps(plan, self.states[i], self.dpdx[i], 0, chunk)
            rem = specs[i].steps % chunk
            tail = GraphedSteps(plan, self.states[i], self.dpdx[i], 0, rem) if rem else None
            self.graphs.append((full, specs[i].steps // chunk, tail))
        torch.cuda.synchronize(self.device)

    @property
    def total_steps(self) -> int:
        return sum(s.steps for s in self.specs)

    def reset(self) -> None:
        for st, init, dp in zip(self.states, self.initial, self.dpdx):
            st.copy_(init)
            dp.zero_()
        torch.cuda.synchronize(self.device)

    def _replay(self, i: int) -> None:
        full, nfull, tail = self.graphs[i]
        for _ in range(nfull):
            full.replay()
        if tail is not None:
            tail.replay()

    def run(self) -> float:
        """All runs to their horizons, overlapped on the stream pool; returns
        the elapsed device time in ms (CUDA events)."""
        main = torch.cuda.current_stream(self.device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(main)
        for s in self.streams:
            s.wait_event(start)
        # longest runs first so the tail is short
        order = sorted(range(len(self.specs)), key=lambda i: -self.specs[i].steps * self.specs[i].ny * self.specs[i].n ** 2)
        for k, i in enumerate(order):
            with torch.cuda.stream(self.streams[k % len(self.streams)]):
                self._replay(i)
        for s in self.streams:
            main.wait_stream(s)
        stop.record(main)
        torch.cuda.synchronize(self.device)
        for plan in self.plans:
            plan.check_device_errors()
        return start.elapsed_time(stop)

    def run_sequential(self, runs: Optional[List[int]] = None) -> float:
        """The same runs one after another on one stream (device time, ms)."""
        main = torch.cuda.current_stream(self.device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(main)
        for i in (runs if runs is not None else range(len(self.specs))):
            self._replay(i)
        stop.record(main)
        torch.cuda.synchronize(self.device)
        for plan in self.plans:
            plan.check_device_errors()
        return start.elapsed_time(stop)

    def energies(self) -> np.ndarray:
        return np.array([p.energy(st).item() for p, st in zip(self.plans, self.states)])


class BatchedEnsemble:
    """The same ensemble with every group of runs that share a box stepped as
    one batch plan: one set of launches per RK stage advances all runs of the
    group (each y-operator is a single product over the group, the transform
    kernels see one plane per (y, run), Re enters per run).

    Runs of a group are ordered by horizon, longest first. The group steps in
    phases between successive horizons; at the end of a phase the runs that
    reached their horizon (the tail of the order) are copied out and the batch
    shrinks (jsd_set_batch_active), so no run steps past its horizon. Each
    phase replays CUDA graphs of up to `chunk` steps; groups are spread over a
    pool of streams.
    """

    def __init__(self, specs: List[RunSpec], streams: int = 4, chunk: int = 100, precision: str = "fp64",
                 device: str = "cuda"):
        from ._plan import pack_runs

        self.specs = specs
        self.device = torch.device(device)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(max(1, streams))]
        keys = {}
        for i, s in enumerate(specs):
            keys.setdefault((s.n, s.ny, s.lx, s.lz, s.dt, s.linearise), []).append(i)
        self.groups = []
        for (n, ny, lx, lz, dt, lin), idx in keys.items():
            idx = sorted(idx, key=lambda i: (-specs[i].steps, i))
            shape = (n, ny, n)
            modes, phys = mode_counts(shape)
            kmax = (min(8, modes[0] // 2), min(8, modes[2] // 2))
            plan = StepPlan(modes, phys, lx, lz, _native.JSD_KIND_PERTURBATION, [specs[i].re for i in idx], dt,
                            linearise=lin, base_u=1 - cheb_points(modes[1]) ** 2, precision=precision,
                            device=device)
            init = pack_runs([seeded_velocity_hat(shape, (lx, lz), kmax, specs[i].e0, specs[i].seed) for i in idx],
                             device=self.device)
            buf = init.clone().reshape(-1)
            dp = torch.zeros(1, dtype=torch.float64, device=self.device)
            mx, _, mz = modes
            # phases: (active runs, steps in the phase, graphs)
            steps = [specs[i].steps for i in idx]
            phases, done = [], 0
            bounds = sorted(set(steps))
            for b in bounds:
                active = sum(1 for st in steps if st >= b)
                phases.append([active, b - done, []])
                done = b
            for ph in phases:
                active, n_steps, graphs = ph
                if n_steps <= 0:
                    continue
                plan.set_batch_active(active)
                view = buf[: 3 * ny * active * mx * mz].view(3, ny, active, mx, mz)
                # the graphs' eager warm-up steps a copy of the view: give it
                # the phase's own layout of valid states (its first runs)
                view.copy_(init[:, :, :active])
                full, rem = divmod(n_steps, chunk)
                if full:
                    graphs.append((GraphedSteps(plan, view, dp, 0, chunk), full))
                if rem:
                    graphs.append((GraphedSteps(plan, view, dp, 0, rem), 1))
            buf.copy_(init.reshape(-1))
            plan.check_device_errors()  # the warm-up steps ran on valid states
            self.groups.append({"idx": idx, "plan": plan, "init": init, "buf": buf, "dp": dp, "phases": phases,
                                "dims": (ny, mx, mz), "final": torch.zeros_like(init)})
        torch.cuda.synchronize(self.device)

    @property
    def total_steps(self) -> int:
        return sum(s.steps for s in self.specs)

    def reset(self) -> None:
        for g in self.groups:
            g["buf"].copy_(g["init"].reshape(-1))
            g["dp"].zero_()
            g["final"].zero_()
        torch.cuda.synchronize(self.device)

    def _run_group(self, g) -> None:
        ny, mx, mz = g["dims"]
        buf, phases = g["buf"], g["phases"]
        for k, (active, n_steps, graphs) in enumerate(phases):
            for graph, reps in graphs:
                for _ in range(reps):
                    graph.replay()
            view = buf[: 3 * ny * active * mx * mz].view(3, ny, active, mx, mz)
            nxt = phases[k + 1][0] if k + 1 < len(phases) else 0
            # runs nxt .. active-1 reached their horizon: keep their states
            g["final"][:, :, nxt:active].copy_(view[:, :, nxt:active])
            if nxt:
                keep = view[:, :, :nxt].clone()
                buf[: 3 * ny * nxt * mx * mz].view(3, ny, nxt, mx, mz).copy_(keep)

    def run(self) -> float:
        """All runs to their horizons; returns the elapsed device time in ms."""
        main = torch.cuda.current_stream(self.device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(main)
        for s in self.streams:
            s.wait_event(start)
        order = sorted(range(len(self.groups)),
                       key=lambda k: -sum(self.specs[i].steps for i in self.groups[k]["idx"]) *
                       self.groups[k]["dims"][0] * self.groups[k]["dims"][1] ** 2)
        for j, k in enumerate(order):
            with torch.cuda.stream(self.streams[j % len(self.streams)]):
                self._run_group(self.groups[k])
        for s in self.streams:
            main.wait_stream(s)
        stop.record(main)
        torch.cuda.synchronize(self.device)
        for g in self.groups:
            g["plan"].check_device_errors()
        return start.elapsed_time(stop)

    def energies(self) -> np.ndarray:
        """Kinetic energy of every run at its horizon, in the order of `specs`."""
        out = np.zeros(len(self.specs))
        for g in self.groups:
            plan = g["plan"]
            plan.set_batch_active(len(g["idx"]))
            e = plan.energy_runs(g["final"]).cpu().numpy()
            for pos, i in enumerate(g["idx"]):
                out[i] = e[pos]
        return out
