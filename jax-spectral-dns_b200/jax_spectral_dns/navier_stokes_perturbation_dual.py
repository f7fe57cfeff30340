"""Dual (adjoint) perturbation equations on the B200 step kernels.

Drop-in for ``NavierStokesVelVortPerturbationDual`` of
dakling/jax-spectral-dns (navier_stokes_perturbation_dual.py:376-1201): the
dual is the same RK3/CN stepper run backward -- Re and dt negated, the
implicit operators taken from the forward equation, the nonlinear term replaced
by the adjoint convection with the forward state u(T - t) frozen over each step
-- started from -u(T). The gradient of the gain G = E(T)/E(0) is
(u0 - v0) / E0.
"""
from __future__ import annotations

from typing import Any, Optional, Tuple

import torch

from . import _native
from ._plan import to_device_layout, to_reference_layout
from .equation import print_verb
from .field import FourierField, VectorField
from .navier_stokes_perturbation import NavierStokesVelVortPerturbation


class NavierStokesVelVortPerturbationDual(NavierStokesVelVortPerturbation):
    name = ("Dual Navier Stokes equation (velocity-vorticity formulation) for perturbations on top of a "
            "base flow.")
    _kind = _native.JSD_KIND_DUAL
    # objectives (..._dual.py:388-400): the gain E(T)/E(0); the gain of the part
    # of u(T) with kx != 0 (gain_3d); the gain of u(T) without its (kx, kz) =
    # (0, 0) mode (gain_no_00); the time-averaged dissipation, whose dual starts
    # from zero and is driven by a source from the forward history
    optimisation_modes = ("gain", "gain_3d", "dissipation", "gain_no_00")

    @staticmethod
    def _objective_part(mode: str, data: torch.Tensor) -> torch.Tensor:
        """The part of a (3, Mx, Ny, Mz) final state the objective measures."""
        if mode == "gain":
            return data
        out = data.clone()
        if mode == "gain_3d":
            out[:, 0] = 0.0  # minus field_2d(0): the kx = 0 modes
        elif mode == "gain_no_00":
            out[:, 0, :, 0] = 0.0  # minus field_2d(0).field_2d(2): the (0, 0) mode
        else:
            out.zero_()  # dissipation: the dual starts from zero
        return out

    def __init__(self, velocity_field: Optional[VectorField], forward_equation: NavierStokesVelVortPerturbation,
                 **params: Any):
        self.epsilon = params.get("epsilon", 1e-5)
        mode = params.get("optimisation_mode", "gain")
        if mode not in self.optimisation_modes:
            raise ValueError(f"unknown optimisation mode {mode!r}. Valid choices are {self.optimisation_modes}")
        self.optimisation_mode = mode
        if params.get("constant_mass_flux", False):
            raise NotImplementedError("the dual with constant mass flux is not supported")
        if velocity_field is None:
            velocity_field = forward_equation.get_latest_field("velocity_hat") * 0.0
        self.forward_equation = forward_equation
        super().__init__(velocity_field, **params)
        self.velocity_u_hat_0 = forward_equation.get_initial_field("velocity_hat")
        self.velocity_field_u_history = None
        self.dPdx_history = None
        self.checkpointing = bool(params.get("checkpointing", False))
        self.gain = None
        self._forward_done = False
        self._backward_done = False

    def get_fixed_params(self):
        return self.forward_equation

    @classmethod
    def FromNavierStokesVelVortPerturbation(cls, nse: NavierStokesVelVortPerturbation, **params: Any):
        """Dual of a forward perturbation problem (..._dual.py:542-589)."""
        nse.write_entire_output = True
        nse.write_intermediate_output = False
        stripped = {k: v for k, v in params.items() if k not in (
            "Re_tau", "Re", "dt", "end_time", "velocity_base_hat", "constant_mass_flux", "linearise",
            "linearise_switch", "coupling_term", "coupling_term_switch")}
        dual = cls(None, nse, Re_tau=-nse.get_Re_tau(), dt=-nse.get_dt(), end_time=-nse.end_time,
                   velocity_base_hat=nse.get_latest_field("velocity_base_hat"),
                   constant_mass_flux=nse.constant_mass_flux, linearise=nse.linearise(0),
                   coupling_term=True, **stripped)
        return dual

    def _plan_spec(self, time_step: int = 0) -> dict:
        """The dual steps with the forward equation's implicit operators
        (positive Re and dt) and -dt on the explicit terms."""
        spec = super()._plan_spec(time_step)
        spec["re_tau"] = self.forward_equation.get_Re_tau()
        spec["dt"] = self.forward_equation.get_dt()
        spec["dt_explicit"] = self.get_dt()
        spec["constant_mass_flux"] = False
        return spec

    def _time_dependent(self) -> bool:
        return self.optimisation_mode == "dissipation" or super()._time_dependent()

    def _prepare_step(self, plan, time_step: int) -> None:
        super()._prepare_step(plan, time_step)
        if self.optimisation_mode == "dissipation":
            plan.set_source(*self._dissipation_source(time_step))

    def _dissipation_source(self, time_step: int):
        """Source of the dissipation objective's dual step `time_step`
        (..._dual.py:962-990): s = -lap(u) / |Re_tau T| of the forward state
        u = history[-1 - time_step], composed as the reference's step adds it
        (navier_stokes.py:1697-1703): with C = (curl s)_y, h_v gains
        i kz C[kx index 0] - i kx_1 C[kx index 2] and h_g gains C[kx index 1],
        each plane added at every kx; the mean flow gains (s_x, s_z) at
        (0, 0) (navier_stokes.py:1461-1491). Returns (h_v, h_g) in the
        device's (Ny, Mx, Mz) layout and the (2 Ny,) mean-flow source."""
        traj = self.forward_equation._trajectory_device
        if traj is None:
            raise RuntimeError("run the forward calculation before the dissipation dual step")
        u = traj[traj.shape[0] - 1 - time_step].permute(0, 2, 1, 3)  # (3, Mx, Ny, Mz)
        dom = self.get_domain()
        scale = -1.0 / abs(self.get_Re_tau() * self.end_time)
        s = torch.stack([(dom.diff(u[i], 0, 2) + dom.diff(u[i], 1, 2) + dom.diff(u[i], 2, 2)) * scale
                         for i in range(3)])
        C = dom.curl(s)[1]
        kx = torch.as_tensor(dom.grid[0], dtype=torch.float64, device=u.device)
        kz = torch.as_tensor(dom.grid[2], dtype=torch.float64, device=u.device)
        hv_plane = 1j * kz * C[0] - 1j * kx[1] * C[2]  # (Ny, Mz)
        mx = u.shape[1]
        hv = hv_plane.unsqueeze(1).expand(-1, mx, -1).contiguous()
        hg = C[1].unsqueeze(1).expand(-1, mx, -1).contiguous()
        s00 = torch.cat([s[0][0, :, 0], s[2][0, :, 0]]).contiguous()
        return hv, hg, s00

    def _prepare_plan_history(self, plan) -> None:
        if self.linearise(0):
            return
        traj = getattr(self.forward_equation, "_trajectory_device", None)
        if traj is None:
            raise RuntimeError("run the forward calculation before the nonlinear dual step")
        if plan._history is not traj:
            plan.set_history(traj)

    def update_with_nse(self) -> None:
        """Forget the previous forward/dual runs after the forward initial field
        changed (..._dual.py:634-641)."""
        self.forward_equation.write_entire_output = True
        self.forward_equation.write_intermediate_output = False
        self.clear_field("velocity_hat")
        self.dPdx = 0.0
        self.forward_equation.dPdx = 0.0
        self.velocity_field_u_history = None
        self.dPdx_history = None
        self._forward_done = False
        self._backward_done = False
        self.forward_equation._trajectory_device = None

    def is_forward_calculation_done(self) -> bool:
        return self._forward_done

    def is_backward_calculation_done(self) -> bool:
        return self._backward_done

    def run_forward_calculation(self) -> None:
        """Forward run keeping the trajectory; dual initial field -u(T)
        (..._dual.py:850-939)."""
        nse = self.forward_equation
        self.velocity_u_hat_0 = nse.get_initial_field("velocity_hat")
        if not self._forward_done:
            nse.set_initial_field("velocity_hat", nse.get_initial_field("velocity_hat"))
            nse.write_entire_output = True
            nse.end_time = -1.0 * self.end_time
            traj, dps, _ = nse.solve_scan()
            self.velocity_field_u_history = traj
            self.dPdx_history = dps
            self._forward_done = True
        # dual initial field: minus the objective's part of u(T) (..._dual.py:904-937)
        uT = nse.get_latest_field("velocity_hat")
        part = self._objective_part(self.optimisation_mode, uT.get_data())
        self.set_initial_field("velocity_hat",
                               VectorField.FromData(FourierField, self.get_physical_domain(), -part,
                                                    name="velocity_hat"))

    def run_backward_calculation(self) -> None:
        if not self._backward_done:
            self.run_forward_calculation()
            self.write_entire_output = False
            self.write_intermediate_output = False
            self.dPdx = 0.0
            print_verb("performing backward (adjoint) calculation...", verbosity_level=2)
            self.solve_scan()
            self._backward_done = True

    def _gain_of(self, mode: str) -> float:
        self.run_forward_calculation()
        nse = self.forward_equation
        e0 = nse.energy_of(nse.get_initial_field("velocity_hat").get_data())
        eT = nse.energy_of(self._objective_part(mode, nse.get_latest_field("velocity_hat").get_data()))
        self.gain = eT / e0
        return self.gain

    def get_gain(self) -> float:
        """E(T) / E(0) (..._dual.py:1058-1063)."""
        return self._gain_of("gain")

    def get_gain_3d(self) -> float:
        """Energy of u(T) without its kx = 0 part over E(0) (..._dual.py:1065-1077)."""
        return self._gain_of("gain_3d")

    def get_gain_no_00(self) -> float:
        """Energy of u(T) without its (0, 0) mode over E(0) (..._dual.py:1079-1091)."""
        return self._gain_of("gain_no_00")

    def get_dissipation_average(self) -> float:
        """(1 / |Re_tau n|) sum over the n stored forward states of
        sum_ij (d_j u_i)^2, the squares taken of the spectral coefficients,
        then no_hat and the volume integral (..._dual.py:1089-1104)."""
        self.run_forward_calculation()
        traj = self.forward_equation._trajectory_device
        dom = self.get_domain()
        acc = None
        for t in range(traj.shape[0]):
            u = traj[t].permute(0, 2, 1, 3)
            for i in range(3):
                for j in range(3):
                    d = dom.diff(u[i], j) ** 2
                    acc = d if acc is None else acc + d
        acc = acc / abs(self.get_Re_tau() * traj.shape[0])
        return FourierField(self.get_physical_domain(), acc).no_hat().volume_integral()

    def get_objective_fun(self) -> float:
        if self.optimisation_mode == "dissipation":
            self.gain = self.get_gain()
            return self.get_dissipation_average()
        return self._gain_of(self.optimisation_mode)

    def get_objective_fun_name(self) -> str:
        return self.optimisation_mode

    def get_grad(self, u_hat_0: Optional[VectorField] = None, v_hat_0: Optional[VectorField] = None):
        """(u0 - v0) / E0 (..._dual.py:1106-1120)."""
        if u_hat_0 is None and v_hat_0 is None:
            self.run_backward_calculation()
        if u_hat_0 is None:
            u_hat_0 = self.forward_equation.get_initial_field("velocity_hat")
        if v_hat_0 is None:
            v_hat_0 = self.get_latest_field("velocity_hat")
        self.get_gain()
        e0 = self.forward_equation.energy_of(u_hat_0.get_data())
        return (u_hat_0.get_data() - v_hat_0.get_data()) / e0

    def _projection(self, step_size, u_hat_0, v_data, step_size_factor):
        """Step along the gradient projected on the constant-energy sphere
        (..._dual.py:1122-1150)."""
        if step_size_factor is None:
            step_size_factor = 0.9
        assert 0 < step_size_factor < 1, "invalid choice of initial step size factor."
        nse = self.forward_equation
        u_data = u_hat_0.get_data()
        e0 = nse.energy_of(u_data)
        e0_adj = nse.energy_of(v_data)
        # 2 <v, u> = E(u + v) - E(u) - E(v) (energy is a quadratic form)
        c0 = nse.energy_of(u_data + v_data) - e0 - e0_adj
        max_step = step_size_factor * (e0_adj / e0 - c0 ** 2 / (4 * e0 ** 2)) ** (-1 / 2)
        step_size = min(step_size, max_step)
        A = (step_size * c0 - 2 * e0) / (2 * step_size * e0)
        lam = A + (A ** 2 - (step_size * e0_adj - c0) / (step_size * e0)) ** 0.5
        return lam, step_size

    def get_projected_grad(self, step_size: float, u_hat_0=None, v_hat_0=None, step_size_factor=None
                           ) -> Tuple[torch.Tensor, bool]:
        if u_hat_0 is None and v_hat_0 is None:
            self.run_backward_calculation()
        if u_hat_0 is None:
            u_hat_0 = self.velocity_u_hat_0
        if v_hat_0 is None:
            v_hat_0 = self.get_latest_field("velocity_hat")
        lam, _ = self._projection(step_size, u_hat_0, v_hat_0.get_data(), step_size_factor)
        return lam * u_hat_0.get_data() - v_hat_0.get_data(), True

    def get_projected_cg_grad(self, step_size: float, beta: float, old_grad, u_hat_0=None, v_hat_0=None,
                              step_size_factor=None) -> Tuple[torch.Tensor, bool]:
        if u_hat_0 is None and v_hat_0 is None:
            self.run_backward_calculation()
        if u_hat_0 is None:
            u_hat_0 = self.velocity_u_hat_0
        if v_hat_0 is None:
            v_hat_0 = self.get_latest_field("velocity_hat")
        v_data = v_hat_0.get_data() - beta * old_grad
        lam, _ = self._projection(step_size, u_hat_0, v_data, step_size_factor)
        return lam * u_hat_0.get_data() + (-1.0 * v_hat_0.get_data() + beta * old_grad), True
