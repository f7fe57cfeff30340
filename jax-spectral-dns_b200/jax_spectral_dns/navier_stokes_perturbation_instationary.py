"""Perturbations about a time-dependent base flow on the B200 step kernels.

Drop-in for ``NavierStokesVelVortPerturbationInstationary`` of
dakling/jax-spectral-dns (navier_stokes_perturbation_instationary.py:28-108):
the base flow is the wall-driven profile U(y, t) of ``vel_base_fn``, with
wall speed g_w(t) = 1 - exp(-kappa t) (``accelerate``) or exp(-kappa t) and
its Fourier-sine correction series of ``n_max`` terms, re-evaluated at every
time step t = time_step * dt; the nonlinear term is the full (not linearised)
skew-symmetric perturbation term with ``coupling_term`` off; the pressure
gradient stays zero. The native plan is shared by all steps and receives
U(y, t) and dU/dy before each step (jsd_set_base_flow).
"""
from __future__ import annotations

from typing import Any

import numpy as np
import torch

from .navier_stokes_perturbation import NavierStokesVelVortPerturbation
from .seeds import cheb_diff_matrix, cheb_points


class NavierStokesVelVortPerturbationInstationary(NavierStokesVelVortPerturbation):
    name = ("Navier Stokes equation (velocity-vorticity formulation) for perturbations on top of a time-dependent "
            "base flow.")

    def __init__(self, velocity_field, **params: Any):
        super().__init__(velocity_field, **params)
        self.kappa = params.get("kappa", 1.0)
        self.accelerate = params.get("accelerate", True)
        self.n_max = params.get("n_max", 100)
        self._base_keep = None

    def base_profile_at(self, time_step: int) -> np.ndarray:
        """U(y) at t = time_step * dt on the Chebyshev points (vel_base_fn)."""
        t = float(np.arange(0, self.end_time, self.get_dt())[time_step])
        re = self.get_Re_tau()
        k = self.kappa
        if self.accelerate:
            gw, dgw, dgw0 = 1.0 - np.exp(-k * t), k * np.exp(-k * t), k
        else:
            gw, dgw, dgw0 = np.exp(-k * t), -k * np.exp(-k * t), -k
        y = cheb_points(self.get_physical_domain().get_shape()[1])
        out = gw * y + re / 6 * dgw * (y ** 3 - y)
        coeff = -1.0 if self.accelerate else 1.0
        for n in range(1, self.n_max):
            c1n = (-2 * re * (-1) ** n / (np.pi * n) ** 3) * dgw0
            a_n = (np.pi * n) ** 2 / re
            integ = k ** 2 * coeff / (a_n - k)
            out = out + (np.exp(-k * t) - np.exp(-a_n * t)) * (
                -(2 * re * (-1) ** n) / (np.pi * n) ** 3 * integ * np.sin(n * np.pi * y))
            out = out + np.exp(-a_n * t) * c1n * np.sin(n * np.pi * y)
        return out

    def set_linearise(self) -> None:
        """Always the full nonlinear term without the coupling term, zero
        pressure gradient (navier_stokes_perturbation_instationary.py:94-108)."""
        self.flow_rate = self.get_flow_rate()
        self.dPdx = 0.0
        self.linearise = lambda _t: False
        self.coupling_term = lambda _t: False

    def update_pressure_gradient(self, vel_new_field_hat=None, dPdx=None) -> float:
        return 0.0

    def _time_dependent(self) -> bool:
        return True

    def _prepare_step(self, plan, time_step: int) -> None:
        u = self.base_profile_at(time_step)
        du = cheb_diff_matrix(cheb_points(len(u))) @ u
        bu = torch.as_tensor(u, dtype=torch.float64, device=plan.device).contiguous()
        bdu = torch.as_tensor(du, dtype=torch.float64, device=plan.device).contiguous()
        plan.set_base_flow(bu, bdu)
        self._base_keep = (bu, bdu)  # alive until the copies on the stream have run
