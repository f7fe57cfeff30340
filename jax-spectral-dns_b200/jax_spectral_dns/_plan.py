"""Device step plan: owns a native jsd_plan and the device buffers around it.

Spectral states handed to the native library use the plane-major layout
(3, Ny, Mx, Mz) complex128; the reference layout (3, Mx, Ny, Mz) is converted
at this boundary (``to_device_layout`` / ``to_reference_layout``).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _native
from ._ops import device_fft_size, fourier_scale, mean_flow_matrices, operator_tables


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def to_device_layout(x, device="cuda") -> torch.Tensor:
    """(3, Mx, Ny, Mz) or (Mx, Ny, Mz) complex -> contiguous (.., Ny, Mx, Mz) on device."""
    t = torch.as_tensor(x)
    if not t.is_complex():
        t = t.to(torch.complex128)
    t = t.to(device=device, dtype=torch.complex128)
    return t.transpose(-3, -2).contiguous()


def to_reference_layout(x: torch.Tensor) -> torch.Tensor:
    return x.transpose(-3, -2).contiguous()


def pack_runs(states, device="cuda") -> torch.Tensor:
    """Reference-layout states (3, Mx, Ny, Mz) of several runs -> the batch
    layout (3, Ny, runs, Mx, Mz) on the device."""
    dev = torch.stack([to_device_layout(x, device=device) for x in states])  # (runs, 3, Ny, Mx, Mz)
    return dev.permute(1, 2, 0, 3, 4).contiguous()


def unpack_runs(state: torch.Tensor) -> list:
    """Batch layout (3, Ny, runs, Mx, Mz) -> list of reference-layout states."""
    return [to_reference_layout(state[:, :, r]) for r in range(state.shape[2])]


def _stream_ptr() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class StepPlan:
    """One native plan for a box, an equation kind and (Re, dt)."""

    def __init__(self, modes, phys_ref, lx, lz, kind, re_tau, dt, dt_explicit=None, linearise=False,
                 constant_mass_flux=False, flow_rate_target=0.0, base_u: Optional[np.ndarray] = None,
                 fft_sizes=None, device="cuda", precision: str = "fp64", autotune: bool = False):
        if not torch.cuda.is_available():
            raise _native.NativeError("the velocity-vorticity step needs a CUDA device")
        self.lib = _native.load()
        mx, ny, mz = (int(m) for m in modes)
        self.modes = (mx, ny, mz)
        self.device = torch.device(device)
        t = operator_tables(ny)
        batch = np.ndim(re_tau) > 0
        re_runs = np.atleast_1d(np.asarray(re_tau, dtype=np.float64))
        self.n_batch = len(re_runs) if batch else 1
        mats = [mean_flow_matrices(ny, float(r), dt) for r in re_runs]
        rhs_ns = np.concatenate([m[0] for m in mats])
        lhs_inv_ns = np.concatenate([m[1] for m in mats])
        self._keep = []

        def arr(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
            self._keep.append(a)
            return _ptr(a)

        d = _native.JsdDesc()
        d.mx, d.ny, d.mz = mx, ny, mz
        d.px_ref, d.pz_ref = int(phys_ref[0]), int(phys_ref[-1])
        px, pz = fft_sizes if fft_sizes is not None else (device_fft_size(mx), device_fft_size(mz))
        d.px_fft, d.pz_fft = int(px), int(pz)
        self.fft_sizes = (int(px), int(pz))
        d.lx, d.lz = float(lx), float(lz)
        d.kind = int(kind)
        d.linearise = int(bool(linearise))
        d.constant_mass_flux = int(bool(constant_mass_flux))
        d.re_tau = float(re_runs[0])
        if batch:
            d.n_batch = self.n_batch
            d.re_tau_batch = arr(re_runs)
        d.dt = float(dt)
        d.dt_explicit = float(dt if dt_explicit is None else dt_explicit)
        d.flow_rate_target = float(flow_rate_target)
        if base_u is not None:
            bu = np.asarray(base_u, dtype=np.float64)
            d.base_u = arr(bu)
            d.base_du = arr(t.D @ bu)
        d.D, d.V, d.Vinv = arr(t.D), arr(t.V), arr(t.Vinv)
        d.lam, d.sgn, d.c0, d.cN = arr(t.lam), arr(t.sgn), arr(t.c0), arr(t.cN)
        d.w0, d.wN, d.y_weights = arr(t.w0), arr(t.wN), arr(t.y_weights)
        d.rhs_ns, d.lhs_inv_ns = arr(rhs_ns), arr(lhs_inv_ns)
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        d.precision = _native.JSD_PRECISION_MIXED if precision == "mixed" else _native.JSD_PRECISION_FP64
        self.precision = precision
        self.desc = d
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _native.check(self.lib.jsd_plan_create(ctypes.byref(d), ctypes.byref(h)), "jsd_plan_create")
        self.handle = h
        if autotune:
            self.autotune()
        self.scale = fourier_scale(lx, lz)
        self._scalar = torch.zeros(4, dtype=torch.float64, device=self.device)
        self._history = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.jsd_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    # --- calls ------------------------------------------------------------
    def workspace_bytes(self) -> int:
        return int(self.lib.jsd_workspace_bytes(self.handle))

    def autotune(self) -> dict:
        """Time every FP64 tensor-core tile configuration at each GEMM call site
        on this plan's sizes and keep the fastest (jsd_autotune)."""
        with torch.cuda.device(self.device):
            _native.check(self.lib.jsd_autotune(self.handle, _stream_ptr()), "jsd_autotune")
            torch.cuda.synchronize(self.device)
        return self.gemm_configs()

    def set_gemm_config(self, site: str, config: int) -> None:
        _native.check(self.lib.jsd_set_gemm_config(self.handle, _native.GEMM_SITES[site], int(config)),
                      "jsd_set_gemm_config")

    def xmid_variant(self):
        """(x-pass variant in use, [autotune ms of variants 0, 1, 2])."""
        times = (ctypes.c_float * 3)()
        v = int(self.lib.jsd_xmid_variant(self.handle, times))
        return v, [float(t) for t in times]

    def set_xmid_variant(self, variant: int) -> None:
        _native.check(self.lib.jsd_set_xmid_variant(self.handle, int(variant)), "jsd_set_xmid_variant")

    def split_kernel(self):
        """(split-TF32 y-derivative kernel in use: 0 mma.sync, 1 tcgen05, -1 FP64 plan;
        [autotune ms of both])."""
        times = (ctypes.c_float * 2)()
        k = int(self.lib.jsd_split_kernel(self.handle, times))
        return k, [float(t) for t in times]

    def set_split_kernel(self, kernel: int) -> None:
        _native.check(self.lib.jsd_set_split_kernel(self.handle, int(kernel)), "jsd_set_split_kernel")

    def split_eig_in(self) -> int:
        """1 when the mixed form's eigenbasis-in products of the nonlinear
        terms run in split TF32, 0 when FP64-accurate, -1 for FP64 plans."""
        return int(self.lib.jsd_split_eig_in(self.handle))

    def set_split_eig_in(self, on: bool) -> None:
        _native.check(self.lib.jsd_set_split_eig_in(self.handle, int(bool(on))), "jsd_set_split_eig_in")

    def eig_kernel(self, site: int):
        """(eigenbasis product kernel at GEMM site 1 or 2: 0 FP64 DMMA, 1 Ozaki
        int8 tensor cores; [autotune ms of the best DMMA tile and of Ozaki])."""
        times = (ctypes.c_float * 2)()
        k = int(self.lib.jsd_eig_kernel(self.handle, int(site), times))
        return k, [float(t) for t in times]

    def set_eig_kernel(self, site: int, kernel: int) -> None:
        _native.check(self.lib.jsd_set_eig_kernel(self.handle, int(site), int(kernel)), "jsd_set_eig_kernel")

    def check_device_errors(self) -> None:
        """Raise DeviceFailure when a kernel of this plan gave up a bounded wait
        or a stage produced a NaN or an infinity since the last check
        (synchronises the current stream; clears the flag)."""
        _native.check(self.lib.jsd_device_error(self.handle, _stream_ptr()), "jsd_device_error",
                      _native.DeviceFailure)

    def set_wait_limit(self, polls: int) -> None:
        """Polls before a pipeline wait of the tcgen05 kernels gives up (0: default)."""
        _native.check(self.lib.jsd_set_wait_limit(self.handle, int(polls)), "jsd_set_wait_limit")

    def wait_limit(self) -> int:
        return int(self.lib.jsd_wait_limit(self.handle))

    def gemm_configs(self) -> dict:
        """{site: (configuration id, [per-configuration autotune ms])}."""
        out = {}
        for name, site in _native.GEMM_SITES.items():
            times = (ctypes.c_float * _native.DGEMM_CONFIGS)()
            cfg = int(self.lib.jsd_gemm_config(self.handle, site, times))
            out[name] = (cfg, [float(t) for t in times])
        return out

    def launches_per_step(self) -> int:
        """Kernel launches per step after the first of a `step` call."""
        return int(self.lib.jsd_launches_per_step(self.handle))

    def launches(self, n_steps: int) -> int:
        """Kernel launches of one `step(state, dpdx, t, n_steps)` call."""
        if n_steps <= 0:
            return 0
        return n_steps * self.launches_per_step() + int(self.lib.jsd_launches_first_step_extra(self.handle))

    def step(self, state: torch.Tensor, dpdx: torch.Tensor, first_step: int, n_steps: int):
        """Advance a device-layout state in place; dpdx is a 1-element float64 device tensor."""
        assert state.is_contiguous() and state.dtype == torch.complex128 and state.device.type == "cuda"
        assert dpdx.dtype == torch.float64 and dpdx.device.type == "cuda"
        _native.check(self.lib.jsd_step(self.handle, ctypes.c_void_p(state.data_ptr()),
                                        ctypes.c_void_p(dpdx.data_ptr()), int(first_step), int(n_steps),
                                        _stream_ptr()), "jsd_step")

    def step_host_stream(self, host_in, host_out, dpdx: torch.Tensor, first_step: int = 0, n_steps: int = 1):
        """Advance host states: each pinned host_in[k] (reference layout
        (3, Mx, Ny, Mz), complex128) by n_steps, the result into the pinned
        host_out[k]. The host->device copy of state k + 1 and the device->host
        copy of state k - 1 run on two copy streams (one per direction, so
        they overlap each other too) while state k steps on the current stream
        (two device buffers each way), so the transfers overlap the steps.
        dpdx is shared and advanced by every state in turn.
        Returns once everything is enqueued; the current stream waits for the
        last copy."""
        n = len(host_in)
        assert len(host_out) == n
        if n == 0:
            return
        dev = dpdx.device
        main = torch.cuda.current_stream(dev)
        if getattr(self, "_copy_streams", None) is None or self._copy_streams[0].device != dev:
            self._copy_streams = (torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev))
        copy, back = self._copy_streams
        shape = tuple(host_in[0].shape)
        din = [torch.empty(shape, dtype=torch.complex128, device=dev) for _ in range(2)]
        dout = [torch.empty(shape, dtype=torch.complex128, device=dev) for _ in range(2)]
        ev = {key: [torch.cuda.Event() for _ in range(2)] for key in ("loaded", "consumed", "computed", "drained")}
        copy.wait_stream(main)  # the buffers were allocated on the current stream
        back.wait_stream(main)

        def load(k):
            b = k % 2
            with torch.cuda.stream(copy):
                if k >= 2:
                    copy.wait_event(ev["consumed"][b])  # state k - 2 has left din[b]
                din[b].copy_(host_in[k], non_blocking=True)
                ev["loaded"][b].record(copy)

        load(0)
        if n > 1:
            load(1)
        for k in range(n):
            b = k % 2
            main.wait_event(ev["loaded"][b])
            st = din[b].transpose(-3, -2).contiguous()
            ev["consumed"][b].record(main)
            if k + 2 < n:
                load(k + 2)
            self.step(st, dpdx, first_step, n_steps)
            if k >= 2:
                main.wait_event(ev["drained"][b])  # state k - 2 has left dout[b]
            dout[b].copy_(st.transpose(-3, -2))
            ev["computed"][b].record(main)
            with torch.cuda.stream(back):
                back.wait_event(ev["computed"][b])
                host_out[k].copy_(dout[b], non_blocking=True)
                ev["drained"][b].record(back)
        main.wait_stream(copy)
        main.wait_stream(back)

    def step_trajectory(self, state: torch.Tensor, dpdx: torch.Tensor, first_step: int, n_steps: int
                        ) -> torch.Tensor:
        """Advance in place and return all states (n_steps + 1, 3, Ny, Mx, Mz)."""
        assert state.is_contiguous() and state.dtype == torch.complex128
        traj = torch.empty((n_steps + 1,) + tuple(state.shape), dtype=state.dtype, device=state.device)
        _native.check(self.lib.jsd_step_trajectory(self.handle, ctypes.c_void_p(state.data_ptr()),
                                                   ctypes.c_void_p(dpdx.data_ptr()), int(first_step), int(n_steps),
                                                   ctypes.c_void_p(traj.data_ptr()), _stream_ptr()),
                      "jsd_step_trajectory")
        return traj

    def step_adjoint(self, cotangent: torch.Tensor, n_steps: int) -> None:
        """Discrete adjoint (linearised perturbation plans): replace the gradient
        with respect to the state after n_steps steps, in place, by the gradient
        with respect to the state before them (jsd_step_adjoint)."""
        assert cotangent.is_contiguous() and cotangent.dtype == torch.complex128 and cotangent.device.type == "cuda"
        _native.check(self.lib.jsd_step_adjoint(self.handle, ctypes.c_void_p(cotangent.data_ptr()), int(n_steps),
                                                _stream_ptr()), "jsd_step_adjoint")

    def energy_grad(self, state: torch.Tensor) -> torch.Tensor:
        """Gradient of energy(state) with respect to the real and imaginary parts
        of the coefficients (device layout, complex128)."""
        out = torch.empty_like(state)
        _native.check(self.lib.jsd_energy_grad(self.handle, ctypes.c_void_p(state.data_ptr()),
                                               ctypes.c_void_p(out.data_ptr()), _stream_ptr()), "jsd_energy_grad")
        return out

    def set_history(self, states: Optional[torch.Tensor]):
        """Forward trajectory (n, 3, Ny, Mx, Mz) for the dual equations."""
        self._history = states
        if states is None:
            _native.check(self.lib.jsd_set_history(self.handle, None, 0), "jsd_set_history")
        else:
            assert states.is_contiguous() and states.dtype == torch.complex128
            _native.check(self.lib.jsd_set_history(self.handle, ctypes.c_void_p(states.data_ptr()),
                                                   int(states.shape[0])), "jsd_set_history")

    def set_source(self, hv: Optional[torch.Tensor] = None, hg: Optional[torch.Tensor] = None,
                   s00: Optional[torch.Tensor] = None):
        """Source terms added in every stage of the following steps: hv, hg
        (Ny, Mx, Mz) complex to the nonlinear terms h_v, h_g and s00 (2 Ny,)
        complex (x then z) to the mean-flow forcing; no arguments switch them
        off. The plan keeps the tensors alive until the next call."""
        if hv is None:
            self._source = None
            _native.check(self.lib.jsd_set_source(self.handle, None, None, None), "jsd_set_source")
            return
        src = tuple(t.contiguous() for t in (hv, hg, s00))
        for t in src:
            assert t.dtype == torch.complex128 and t.is_cuda
        assert src[0].numel() == src[1].numel() == self.modes[1] * self.modes[0] * self.modes[2]
        assert src[2].numel() == 2 * self.modes[1]
        self._source = src
        _native.check(self.lib.jsd_set_source(self.handle, *(ctypes.c_void_p(t.data_ptr()) for t in src)),
                      "jsd_set_source")

    def energy(self, state: torch.Tensor) -> torch.Tensor:
        out = torch.empty(1, dtype=torch.float64, device=state.device)
        _native.check(self.lib.jsd_energy(self.handle, ctypes.c_void_p(state.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), _stream_ptr()), "jsd_energy")
        return out

    def energy_runs(self, state: torch.Tensor) -> torch.Tensor:
        """Energies of the active runs of a batch plan (device tensor)."""
        out = torch.empty(self.batch_active(), dtype=torch.float64, device=state.device)
        _native.check(self.lib.jsd_energy_runs(self.handle, ctypes.c_void_p(state.data_ptr()),
                                               ctypes.c_void_p(out.data_ptr()), _stream_ptr()), "jsd_energy_runs")
        return out

    def set_coupling_term(self, on: bool) -> None:
        _native.check(self.lib.jsd_set_coupling_term(self.handle, int(bool(on))), "jsd_set_coupling_term")

    def set_base_flow(self, base_u: torch.Tensor, base_du: torch.Tensor) -> None:
        """U(y) and dU/dy as float64 device tensors of Ny entries (copied on the current stream)."""
        assert base_u.dtype == torch.float64 and base_du.dtype == torch.float64
        assert base_u.is_contiguous() and base_du.is_contiguous()
        _native.check(self.lib.jsd_set_base_flow(self.handle, ctypes.c_void_p(base_u.data_ptr()),
                                                 ctypes.c_void_p(base_du.data_ptr()), _stream_ptr()),
                      "jsd_set_base_flow")

    def set_batch_active(self, n_runs: int) -> None:
        _native.check(self.lib.jsd_set_batch_active(self.handle, int(n_runs)), "jsd_set_batch_active")

    def batch_active(self) -> int:
        return int(self.lib.jsd_batch_active(self.handle))

    def flow_rate(self, u_field: torch.Tensor) -> torch.Tensor:
        out = torch.empty(1, dtype=torch.float64, device=u_field.device)
        _native.check(self.lib.jsd_flow_rate(self.handle, ctypes.c_void_p(u_field.data_ptr()),
                                             ctypes.c_void_p(out.data_ptr()), _stream_ptr()), "jsd_flow_rate")
        return out

    def correct_mass_flux(self, state: torch.Tensor, dpdx: Optional[torch.Tensor] = None):
        _native.check(self.lib.jsd_correct_mass_flux(
            self.handle, ctypes.c_void_p(state.data_ptr()),
            ctypes.c_void_p(dpdx.data_ptr()) if dpdx is not None else None, _stream_ptr()),
            "jsd_correct_mass_flux")

    def profile(self, enable: bool) -> None:
        _native.check(self.lib.jsd_profile_enable(self.handle, int(bool(enable))), "jsd_profile_enable")

    def profile_read(self, name: str):
        """(total ms, launches, algorithmic work) of one kernel class since the last read."""
        ms, n, w = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
        _native.check(self.lib.jsd_profile_read(self.handle, _native.PROF_CLASSES[name], ctypes.byref(ms),
                                                ctypes.byref(n), ctypes.byref(w)), "jsd_profile_read")
        return ms.value, n.value, w.value

    def nonlinear_terms(self, state: torch.Tensor, time_step: int = 0):
        mx, ny, mz = self.modes
        hv = torch.empty((ny, mx, mz), dtype=torch.complex128, device=state.device)
        hg = torch.empty_like(hv)
        _native.check(self.lib.jsd_nonlinear_terms(self.handle, ctypes.c_void_p(state.data_ptr()), int(time_step),
                                                   ctypes.c_void_p(hv.data_ptr()), ctypes.c_void_p(hg.data_ptr()),
                                                   _stream_ptr()), "jsd_nonlinear_terms")
        return hv, hg


class GraphedSteps:
    """n_steps of a plan on fixed device buffers captured in one CUDA graph.

    ``jsd_step`` launches only on the caller's stream and allocates nothing,
    so the whole loop (33 launches per step at the benchmark size) is recorded
    once and replayed with a single launch. The captured buffers (state,
    dpdx, the optional trajectory output and any registered dual history)
    must stay alive and in place; ``replay`` advances them exactly as the
    same ``step`` call would.
    """

    def __init__(self, plan: StepPlan, state: torch.Tensor, dpdx: torch.Tensor, first_step: int, n_steps: int,
                 trajectory: Optional[torch.Tensor] = None):
        self.plan, self.state, self.dpdx, self.trajectory = plan, state, dpdx, trajectory
        # one eager run on copies first, so every kernel is loaded before capture
        ws, wd = state.clone(), dpdx.clone()
        if trajectory is None:
            plan.step(ws, wd, first_step, n_steps)
        else:
            plan.step_trajectory(ws, wd, first_step, n_steps)
        torch.cuda.synchronize(state.device)
        self.graph = torch.cuda.CUDAGraph()
        stream = torch.cuda.Stream(device=state.device)
        stream.wait_stream(torch.cuda.current_stream(state.device))
        with torch.cuda.stream(stream):
            with torch.cuda.graph(self.graph, stream=stream):
                if trajectory is None:
                    plan.step(state, dpdx, first_step, n_steps)
                else:
                    _native.check(plan.lib.jsd_step_trajectory(
                        plan.handle, ctypes.c_void_p(state.data_ptr()), ctypes.c_void_p(dpdx.data_ptr()),
                        int(first_step), int(n_steps), ctypes.c_void_p(trajectory.data_ptr()), _stream_ptr()),
                        "jsd_step_trajectory")
        torch.cuda.current_stream(state.device).wait_stream(stream)

    def replay(self) -> None:
        self.graph.replay()
