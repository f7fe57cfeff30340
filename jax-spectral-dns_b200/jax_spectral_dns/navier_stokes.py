"""Velocity-vorticity Navier-Stokes channel solver on the B200 step kernels.

Drop-in for ``jax_spectral_dns.navier_stokes.NavierStokesVelVort`` of
dakling/jax-spectral-dns (navier_stokes.py:310-2013): same constructor
parameters (Re or Re_tau with u_max_over_u_tau, dt, end_time,
constant_mass_flux), the same ``perform_time_step(vel_hat_data, dPdx,
time_step) -> (vel_hat_data, dPdx)`` contract on (3, Mx, Ny, Mz) complex128
spectral data, ``solve()`` / ``solve_scan()`` over int(end_time / dt) steps,
and the same initial pressure gradient and flow-rate bookkeeping. The RK3 /
Crank-Nicolson step itself runs in the native library (libjsd.so).
"""
from __future__ import annotations

from typing import Any, List, Optional, Tuple

import numpy as np
import torch

from . import _native
from ._plan import StepPlan, to_device_layout, to_reference_layout
from .domain import PhysicalDomain
from .equation import Equation, print_verb
from .field import Field, FourierField, PhysicalField, VectorField


class NavierStokesVelVort(Equation):
    name = "Navier Stokes equation (velocity-vorticity formulation)"
    _kind = _native.JSD_KIND_NS
    max_cfl = 0.7

    def __init__(self, velocity_field: VectorField, **params: Any):
        if "physical_domain" in params:
            physical_domain = params["physical_domain"]
        else:
            physical_domain = velocity_field[0].physical_domain
        domain = physical_domain.hat()
        self._physical_domain: PhysicalDomain = physical_domain
        self._params = dict(params)
        # the CFL limit of the step's fixed parameters (navier_stokes.py:321); the
        # class attribute max_cfl (0.5 for perturbations) is what the solvers read
        self._max_cfl = params.get("max_cfl", 0.7)
        self.u_max_over_u_tau = float(params.get("u_max_over_u_tau", 1.0))
        self.Re_tau = self._re_tau_from(params)
        velocity_field.set_name("velocity_hat")
        super().__init__(domain, velocity_field, **params)
        self._plan: Optional[StepPlan] = None
        self._plan_key = None
        self._plans = {}  # plans by specification (linearise / coupling may change with the step)
        self.enforce_base = False
        self.constant_mass_flux = bool(params.get("constant_mass_flux", False))
        self.flow_rate = self.get_flow_rate()
        if self.constant_mass_flux:
            self.dPdx = -self.flow_rate * 3 / 2 / self.get_Re_tau()
        else:
            self.dPdx = -1.0
        self.number_of_time_steps = 0
        self.nonlinear_update_fn = lambda vel, t: self.nonlinear_terms(vel, t)

    # ---- parameters (navier_stokes.py:661-690) ---------------------------
    def _re_tau_from(self, params) -> float:
        if "Re_tau" in params:
            return float(params["Re_tau"])
        if "Re" in params:
            return float(params["Re"]) / self.u_max_over_u_tau
        raise Exception("Either Re or Re_tau has to be given as a parameter.")

    def get_Re_tau(self, **params) -> float:
        return self.Re_tau

    def get_u_max_over_u_tau(self, **params) -> float:
        return self.u_max_over_u_tau

    def get_max_cfl(self) -> float:
        return self._max_cfl

    def get_number_of_rk_steps(self) -> int:
        return 3

    def get_rk_parameters(self, n_steps: Optional[int] = None):
        """RK3/CN coefficients (navier_stokes.py:898-918)."""
        return ([29 / 96, -3 / 40, 1 / 6], [37 / 160, 5 / 24, 1 / 6], [8 / 15, 5 / 12, 3 / 4],
                [0, -17 / 60, -5 / 12])

    def get_physical_domain(self) -> PhysicalDomain:
        return self._physical_domain

    @classmethod
    def FromVelocityField(cls, velocity_field: VectorField, **params: Any):
        vel_hat = velocity_field.hat()
        vel_hat.set_name("velocity_hat")
        return cls(vel_hat, **params)

    @classmethod
    def FromDomain(cls, domain: PhysicalDomain, **params: Any):
        vel = VectorField([PhysicalField.Zeros(domain) for _ in range(3)], "velocity")
        return cls.FromVelocityField(vel, **params)

    # ---- seeding: (v, omega_y) -> (u, v, w) -------------------------------
    @staticmethod
    def _wall_projection(ny: int, m: int) -> np.ndarray:
        """Least-squares projection, on the Ny Gauss-Lobatto points, onto the
        span of phi_n = T_{n+4} - a_n T_{n+2} - b_n T_n (n < m), a_n =
        2(n+2)/(n+1), b_n = -(n+3)/(n+1), the Chebyshev combinations with
        phi(+-1) = phi'(+-1) = 0 (navier_stokes.py:1027-1060)."""
        key = (ny, m)
        cache = NavierStokesVelVort.__dict__.get("_projections")
        if cache is None:
            cache = {}
            NavierStokesVelVort._projections = cache
        if key not in cache:
            from .domain import get_cheb_grid
            ys = get_cheb_grid(ny)
            basis = np.empty((ny, m))
            for n in range(m):
                coef = np.zeros(n + 5)
                coef[n + 4] = 1.0
                coef[n + 2] = -(2 * (n + 2)) / (n + 1)
                coef[n] = (n + 3) / (n + 1)
                basis[:, n] = np.polynomial.chebyshev.Chebyshev(coef)(ys)
            cache[key] = basis @ np.linalg.lstsq(basis, np.eye(ny), rcond=None)[0]
        return cache[key]

    @classmethod
    def smooth_and_enforce_bc_vel_y(cls, physical_domain: PhysicalDomain, vel_y_slice, M: Optional[int] = None):
        """v projected (least squares on the collocation points) onto profiles
        with v = dv/dy = 0 at both walls, along the first axis
        (navier_stokes.py:1027-1060)."""
        x = torch.as_tensor(vel_y_slice)
        ny = x.shape[0]
        p = torch.as_tensor(cls._wall_projection(ny, ny - 4 if M is None else int(M)), device=x.device)
        return torch.tensordot(p.to(x.dtype), x, dims=([1], [0]))

    @classmethod
    def vort_yvel_to_vel(cls, physical_domain: PhysicalDomain, vort, vel_y, vel_x_00, vel_z_00,
                         two_d: bool = False) -> torch.Tensor:
        """(3, Mx, Ny, Mz) velocity from spectral omega_y and v: v smoothed onto
        the wall-conforming profiles, u and w from continuity and the
        definition of omega_y, u = (-i kx dv/dy + i kz omega_y) / -(kx^2 + kz^2),
        w = (-i kz dv/dy - i kx omega_y) / -(kx^2 + kz^2); the (0,0) mode takes
        vel_x_00, the smoothed v and vel_z_00 (navier_stokes.py:1062-1203).
        With two_d, omega_y and w are zero and, as in the reference, every kz
        column is treated as kz = 0: the whole kx = 0 row takes the (0,0) values
        (u = vel_x_00, v = the smoothed (0,0) profile). All wavenumbers in one
        batched product on the fields' device."""
        vy = torch.as_tensor(vel_y).to(torch.complex128)
        dev = vy.device
        om = torch.zeros_like(vy) if two_d else torch.as_tensor(vort, device=dev).to(torch.complex128)
        fd = physical_domain.hat()
        ny = vy.shape[1]
        proj = torch.as_tensor(cls._wall_projection(ny, ny - 4), device=dev).to(torch.complex128)
        dmat = torch.as_tensor(fd.diff_mats[1], device=dev).to(torch.complex128)
        vs = torch.einsum("lj,ijk->ilk", proj, vy)
        dv = torch.einsum("lj,ijk->ilk", dmat, vs)
        kx = torch.as_tensor(np.asarray(fd.grid[0]), dtype=torch.float64, device=dev)[:, None, None]
        kz = torch.as_tensor(np.asarray(fd.grid[2]), dtype=torch.float64, device=dev)[None, None, :]
        if two_d:
            kz = torch.zeros_like(kz)
        den = -(kx ** 2 + kz ** 2)
        den = torch.where(den == 0, torch.ones_like(den), den)  # the (0,0) columns are replaced below
        u = (-(1j * kx) * dv + (1j * kz) * om) / den
        w = torch.zeros_like(u) if two_d else (-(1j * kz) * dv - (1j * kx) * om) / den
        ux00 = torch.as_tensor(vel_x_00, device=dev).to(torch.complex128)
        if two_d:
            u[0] = ux00[:, None]
            vs[0] = vs[0, :, 0].clone()[:, None]
        else:
            u[0, :, 0] = ux00
            w[0, :, 0] = torch.as_tensor(vel_z_00, device=dev).to(torch.complex128)
        return torch.stack([u, vs, w])

    def update_dt(self, new_dt: float) -> None:
        self._dt = float(new_dt)
        self._plan = None
        self._plans = {}

    # ---- native plan ------------------------------------------------------
    def _plan_spec(self, time_step: int = 0) -> dict:
        dom = self.get_physical_domain()
        return dict(kind=self._kind, re_tau=self.get_Re_tau(), dt=self.get_dt(), dt_explicit=None,
                    linearise=False, constant_mass_flux=self.constant_mass_flux,
                    flow_rate_target=float(self.flow_rate) if self.constant_mass_flux else 0.0,
                    base_u=None, modes=dom.get_shape(), phys=dom.get_shape_aliasing(),
                    lx=dom.scale_factors[0], lz=dom.scale_factors[2])

    def get_plan(self, time_step: int = 0) -> StepPlan:
        """The native plan for time step `time_step` (one per distinct set of
        operators and term switches, created on first use)."""
        spec = self._plan_spec(time_step)
        key = tuple((k, (tuple(v) if isinstance(v, (tuple, list, np.ndarray)) else v)) for k, v in spec.items())
        plan = self._plans.get(key)
        if plan is None:
            plan = StepPlan(spec["modes"], spec["phys"], spec["lx"], spec["lz"], spec["kind"], spec["re_tau"],
                            spec["dt"], dt_explicit=spec["dt_explicit"], linearise=spec["linearise"],
                            constant_mass_flux=spec["constant_mass_flux"],
                            flow_rate_target=spec["flow_rate_target"], base_u=spec["base_u"])
            if not spec.get("coupling", True):
                plan.set_coupling_term(False)
            self._plans[key] = plan
        self._plan, self._plan_key = plan, key
        return plan

    def _time_dependent(self) -> bool:
        """True when the step depends on the step index beyond the dual
        history (term switches, a time-dependent base flow)."""
        return False

    def _prepare_step(self, plan: StepPlan, time_step: int) -> None:
        """Hook run before each step (time-dependent base flows)."""

    def _prepare_plan_history(self, plan: StepPlan) -> None:
        """Hook for the dual equations (forward trajectory)."""

    # ---- flow rate / mass flux (navier_stokes.py:709-805) ---------------
    def get_flow_rate(self, vel_new_field_hat=None) -> float:
        """y-integral of the streamwise velocity at x = z = 0."""
        if vel_new_field_hat is None:
            u_hat = self.get_latest_field("velocity_hat")[0].data
        else:
            u_hat = torch.as_tensor(vel_new_field_hat)[0]
        dom = self.get_physical_domain()
        fd = dom.hat()
        u = fd.field_no_hat(u_hat.to(torch.complex128))
        w = torch.as_tensor(dom.y_weights(), dtype=torch.float64, device=u.device)
        return float(u[0, :, 0] @ w)

    def update_velocity_field_data(self, vel_new_hat_field):
        """u <- hat(no_hat(u) - (Q - Q0)/2) with the native kernel."""
        if not self.constant_mass_flux:
            return vel_new_hat_field
        plan = self.get_plan()
        st = to_device_layout(vel_new_hat_field)
        plan.correct_mass_flux(st, None)
        return to_reference_layout(st)

    def update_velocity_field(self, vel_new_hat: VectorField) -> VectorField:
        if not self.constant_mass_flux:
            return vel_new_hat
        data = self.update_velocity_field_data(vel_new_hat.get_data())
        return VectorField.FromData(FourierField, self.get_physical_domain(), data, name="velocity_hat")

    # ---- stepping ---------------------------------------------------------
    def _make_vf(self, data_ref_layout: torch.Tensor, time_step: int) -> VectorField:
        vf = VectorField.FromData(FourierField, self.get_physical_domain(), data_ref_layout, name="velocity_hat")
        vf.set_time_step(time_step)
        return vf

    def perform_runge_kutta_step(self, vel_hat_data, dPdx, time_step: int):
        plan = self.get_plan(time_step)
        self._prepare_plan_history(plan)
        self._prepare_step(plan, time_step)
        st = to_device_layout(vel_hat_data)
        dp = torch.tensor([float(dPdx)], dtype=torch.float64, device=st.device)
        plan.step(st, dp, int(time_step), 1)
        plan.check_device_errors()
        return to_reference_layout(st), float(dp.item())

    def perform_time_step(self, vel_hat_data=None, dPdx=None, time_step: Optional[int] = None
                          ) -> Tuple[torch.Tensor, float]:
        """One RK3/CN step (navier_stokes.py:1778-1813)."""
        from_fields = vel_hat_data is None
        if from_fields:
            vel_hat_data = self.get_latest_field("velocity_hat").get_data()
        if dPdx is None:
            dPdx = self.dPdx
        assert time_step is not None
        out, dp = self.perform_runge_kutta_step(vel_hat_data, dPdx, time_step)
        if from_fields:
            vf = self._make_vf(out, self.get_latest_field("velocity_hat").get_time_step() + 1)
            self.append_field("velocity_hat", vf, in_place=False)
            self.dPdx = dp
        return out, dp

    def number_of_steps(self) -> int:
        return max(0, int(self.end_time / self.get_dt()))

    def run_device(self, state: torch.Tensor, dpdx: torch.Tensor, first_step: int, n_steps: int,
                   keep_trajectory: bool = False):
        """Advance a device-layout state; optionally return all states
        (n_steps + 1, 3, Ny, Mx, Mz) including the initial one."""
        plan = self.get_plan(first_step)
        self._prepare_plan_history(plan)
        used = {id(plan): plan}
        out = self._run_device(plan, used, state, dpdx, first_step, n_steps, keep_trajectory)
        # the results are visible to the caller from here on: raise if a
        # kernel gave up a bounded wait or the state became non-finite
        for p in used.values():
            p.check_device_errors()
        return out

    def _run_device(self, plan, used, state, dpdx, first_step, n_steps, keep_trajectory):
        if self._time_dependent():
            traj = dps = None
            if keep_trajectory:
                traj = torch.empty((n_steps + 1,) + tuple(state.shape), dtype=state.dtype, device=state.device)
                dps = torch.empty(n_steps + 1, dtype=torch.float64, device=state.device)
                traj[0].copy_(state)
                dps[0] = dpdx[0]
            for t in range(n_steps):
                plan = self.get_plan(first_step + t)
                used[id(plan)] = plan
                self._prepare_plan_history(plan)
                self._prepare_step(plan, first_step + t)
                plan.step(state, dpdx, first_step + t, 1)
                if keep_trajectory:
                    traj[t + 1].copy_(state)
                    dps[t + 1] = dpdx[0]
            return traj, dps
        if not keep_trajectory:
            plan.step(state, dpdx, first_step, n_steps)
            return None, None
        if not plan.desc.constant_mass_flux:
            traj = plan.step_trajectory(state, dpdx, first_step, n_steps)
            return traj, dpdx.expand(n_steps + 1).clone()
        traj = torch.empty((n_steps + 1,) + tuple(state.shape), dtype=state.dtype, device=state.device)
        dps = torch.empty(n_steps + 1, dtype=torch.float64, device=state.device)
        traj[0].copy_(state)
        dps[0] = dpdx[0]
        for t in range(n_steps):
            plan.step(state, dpdx, first_step + t, 1)
            traj[t + 1].copy_(state)
            dps[t + 1] = dpdx[0]
        return traj, dps

    def solve_scan(self):
        """All int(end_time/dt) steps on the device (navier_stokes.py:1826-2013).
        Returns (trajectory, dPdx history, number of steps); the trajectory
        holds every state when write_entire_output or
        write_intermediate_output is set, else only the final state."""
        u0 = self.get_initial_field("velocity_hat").get_data()
        dpdx = self.dPdx
        self.dPdx = 0.0
        n = self.number_of_steps()
        self.number_of_time_steps = n
        self.number_of_outer_steps = n
        self.number_of_inner_steps = 1
        start = self.get_initial_field("velocity_hat").get_time_step()
        st = to_device_layout(u0)
        dp = torch.tensor([float(dpdx)], dtype=torch.float64, device=st.device)
        keep = self.write_entire_output or self.write_intermediate_output
        traj, dps = self.run_device(st, dp, 0, n, keep_trajectory=keep)
        self._trajectory_device = traj
        final = to_reference_layout(st)
        self.append_field("velocity_hat", self._make_vf(final, start + n), in_place=False)
        if keep:
            out = to_reference_layout(traj)
            return out, [float(x) for x in dps[1:].tolist()], n
        return final.unsqueeze(0), [float(dp.item())], n

    def nonlinear_terms(self, vel_hat_data, time_step: int = 0):
        """Nonlinear hook (navier_stokes.py:324-332): (h_v, h_g, vort, None)
        for (3, Mx, Ny, Mz) spectral data, computed by the native kernels."""
        plan = self.get_plan()
        self._prepare_plan_history(plan)
        st = to_device_layout(vel_hat_data)
        hv, hg = plan.nonlinear_terms(st, time_step)
        vort = self.get_domain().curl(torch.as_tensor(vel_hat_data, device=st.device))
        return to_reference_layout(hv), to_reference_layout(hg), vort, None

    def energy_of(self, vel_hat_data) -> float:
        """Kinetic energy of spectral data through the native reduction
        (equal to VectorField.no_hat().energy())."""
        plan = self.get_plan()
        return float(plan.energy(to_device_layout(vel_hat_data)).item())

    def get_cfl(self, i: int = -1):
        vel = self.get_field("velocity_hat", i).no_hat()
        dom = self.get_physical_domain()
        d = [np.diff(dom.grid[k]) for k in range(3)]
        DX, DY, DZ = np.meshgrid(*d, indexing="ij")
        out = []
        for k, DD in enumerate((DX, DY, DZ)):
            V = vel[k].data[1:, 1:, 1:].abs().cpu().numpy()
            with np.errstate(divide="ignore"):
                out.append(float((np.abs(DD) / V).min()))
        return self.get_dt() / np.array(out)

    def post_process(self) -> None:
        if self.post_process_fn is not None:
            for i in range(self.get_number_of_fields("velocity_hat")):
                self.post_process_fn(self, i)
