"""Perturbation equations about a base flow U(y) on the B200 step kernels.

Drop-in for ``NavierStokesVelVortPerturbation`` of dakling/jax-spectral-dns
(navier_stokes_perturbation.py:341-520): the default base flow is
u_max_over_u_tau * (1 - y^2); ``velocity_base_hat`` may supply another
streamwise profile U(y); ``linearise`` drops the quadratic term and
``coupling_term=False`` adds the reference's extra h_g term, both also
switchable at a fraction of the run (``linearise_switch``,
``coupling_term_switch``); ``constant_mass_flux`` keeps zero perturbation
flow rate.
"""
from __future__ import annotations

from typing import Any

import numpy as np
import torch

from . import _native
from .field import FourierField, PhysicalField, VectorField
from .equation import print_verb
from .navier_stokes import NavierStokesVelVort


class NavierStokesVelVortPerturbation(NavierStokesVelVort):
    name = ("Navier Stokes equation (velocity-vorticity formulation) for perturbations on top of a base flow.")
    max_cfl = 0.5
    max_dt = 2e-2
    _kind = _native.JSD_KIND_PERTURBATION

    def __init__(self, velocity_field: VectorField, **params: Any):
        super().__init__(velocity_field, **params)
        dom = self.get_physical_domain()
        if "velocity_base_hat" in params and params["velocity_base_hat"] is not None:
            base_hat = params["velocity_base_hat"]
        else:
            umax = self.get_u_max_over_u_tau()
            ux = PhysicalField.FromFunc(dom, lambda X: umax * (1 - X[1] ** 2) + 0.0 * X[0] * X[2],
                                        name="velocity_x_base")
            zero = PhysicalField.FromFunc(dom, lambda X: 0.0 * X[0] * X[1] * X[2])
            base_hat = VectorField([ux.hat(), zero.hat(), zero.hat()], "velocity_base_hat")
        self.add_field("velocity_base_hat", base_hat)
        self.base_profile = self._base_profile(base_hat)
        # linearise / coupling_term, constant or switched at a fraction of the
        # run (navier_stokes_perturbation.py:385-415)
        n_total = len(np.arange(0, self.end_time, self.get_dt()))
        self.linearise_switch = params.get("linearise_switch")
        if self.linearise_switch is not None:
            assert params.get("linearise") is None, "need to either pass linearise or linearise_switch."
            ls = float(self.linearise_switch)
            self.linearise = lambda t: t < n_total * ls
        else:
            lin = bool(params.get("linearise", False))
            self.linearise = lambda _t: lin
        self.coupling_term_switch = params.get("coupling_term_switch")
        if self.coupling_term_switch is not None:
            assert params.get("coupling_term") is None, "need to either pass coupling_term or coupling_term_switch."
            cs = float(self.coupling_term_switch)
            self.coupling_term = lambda t: not (t < n_total * cs)
        else:
            cpl = bool(params.get("coupling_term", True))
            self.coupling_term = lambda _t: cpl
        self.enforce_base = bool(params.get("enforce_base", False))
        if self.enforce_base:
            raise NotImplementedError("enforce_base is not supported")
        self.set_linearise()

    def _base_profile(self, base_hat: VectorField) -> np.ndarray:
        """U(y) of a streamwise base flow that depends on y only."""
        data = base_hat.get_data()
        mx, ny, mz = data.shape[1:]
        scale = torch.linalg.norm(data).item()
        off = data.clone()
        off[0, 0, :, 0] = 0.0
        if scale > 0 and torch.linalg.norm(off).item() > 1e-12 * scale:
            raise NotImplementedError("only streamwise base flows U(y) are supported")
        u = self.get_physical_domain().hat().field_no_hat(data[0])
        return u[0, :, 0].double().cpu().numpy().copy()

    def _plan_spec(self, time_step: int = 0) -> dict:
        spec = super()._plan_spec(time_step)
        spec["linearise"] = bool(self.linearise(time_step))
        spec["coupling"] = bool(self.coupling_term(time_step))
        spec["base_u"] = self.base_profile
        return spec

    def _time_dependent(self) -> bool:
        return self.linearise_switch is not None or self.coupling_term_switch is not None

    def set_linearise(self) -> None:
        """Pressure-gradient / mass-flux set-up (navier_stokes_perturbation.py:468-520)."""
        if self.constant_mass_flux:
            self.flow_rate = 0.0
            self.dPdx = 0.0
            v0 = self.update_velocity_field(self.get_initial_field("velocity_hat"))
            self.set_initial_field("velocity_hat", v0)
        else:
            self.flow_rate = self.get_flow_rate()
            self.dPdx = 0.0

    def update_pressure_gradient(self, vel_new_field_hat=None, dPdx=None) -> float:
        dp = self.dPdx if dPdx is None else dPdx
        if self.constant_mass_flux:
            dp = dp + self.get_flow_rate(vel_new_field_hat) / self.get_dt()
        return float(dp)
