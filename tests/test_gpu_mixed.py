"""Mixed-precision step: FP32 transforms and products, split-TF32 tensor-core
y-derivatives, FP64 solves. Its error against the FP64 path is what it
reports; the bars here are FP32-level agreement with the reference fixtures
and the energy-history bar of the mixed form (relative energy error <= 1e-6
against FP64)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, turbulent_channel_hat

pytestmark = pytest.mark.gpu


def _run(plan, u0, n, dpdx0=0.0):
    st = to_device_layout(u0)
    dp = torch.tensor([dpdx0], dtype=torch.float64, device="cuda")
    plan.step(st, dp, 0, n)
    return st, dp


def test_mixed_nonlinear_perturbation_vs_reference(cuda):
    d = golden("nonlin_pert_9x33x9")
    modes, phys = mode_counts(tuple(d["shape"]))
    p = StepPlan(modes, phys, *d["lengths"], 1, float(d["re"]), float(d["dt"]),
                 base_u=1 - cheb_points(modes[1]) ** 2, precision="mixed")
    st, _ = _run(p, d["u0"], 20)
    assert rel(to_reference_layout(st).cpu().numpy(), d["u20"]) < 1e-5


def test_mixed_channel_constant_mass_flux_vs_reference(cuda):
    d = golden("ns_cmf_9x33x9")
    modes, phys = mode_counts(tuple(d["shape"]))
    probe = StepPlan(modes, phys, *d["lengths"], 0, float(d["re_tau"]), float(d["dt"]))
    q0 = probe.flow_rate(to_device_layout(d["u0"])[0]).item()
    p = StepPlan(modes, phys, *d["lengths"], 0, float(d["re_tau"]), float(d["dt"]), constant_mass_flux=True,
                 flow_rate_target=q0, precision="mixed")
    st, dp = _run(p, d["u0"], 10, float(d["dpdx"][0]))
    assert rel(to_reference_layout(st).cpu().numpy(), d["u10"]) < 1e-5


def test_mixed_energy_history_128_1000_steps(cuda):
    """The benchmark workload (128x129x128 channel, Re_tau = 180, dt = 0.002,
    constant mass flux, bench.py's seeded field), 1000 steps in both forms
    with the mixed form on its tensor-core kernels: the relative energy error
    of the mixed form against the FP64 form stays below 1e-6 at every 50th
    step and after the last (the bar the mixed form is held to), and the mean
    profile u_00(y) agrees to 1e-6."""
    shape, lx, lz, re_tau = (128, 129, 128), 4 * np.pi, 4 * np.pi / 3, 180.0
    modes, phys = mode_counts(shape)
    u0 = turbulent_channel_hat(shape, (lx, lz), re_tau, (16, 16), seed=0)
    probe = StepPlan(modes, phys, lx, lz, 0, re_tau, 0.002)
    q0 = probe.flow_rate(to_device_layout(u0)[0]).item()
    del probe
    plans = {pr: StepPlan(modes, phys, lx, lz, 0, re_tau, 0.002, constant_mass_flux=True, flow_rate_target=q0,
                          precision=pr) for pr in ("fp64", "mixed")}
    assert plans["mixed"].split_kernel()[0] == 1
    assert all(plans["mixed"].eig_kernel(site)[0] == 1 for site in (1, 2))
    st = {pr: to_device_layout(u0) for pr in plans}
    dp = {pr: torch.tensor([-q0 * 1.5 / re_tau], dtype=torch.float64, device="cuda") for pr in plans}
    worst = 0.0
    for k in range(20):
        e = {}
        for pr, p in plans.items():
            p.step(st[pr], dp[pr], 50 * k, 50)
            e[pr] = p.energy(st[pr]).item()
        worst = max(worst, abs(e["mixed"] / e["fp64"] - 1))
    for p in plans.values():
        p.check_device_errors()
    assert worst < 1e-6, worst
    prof = {pr: to_reference_layout(st[pr])[0, 0, :, 0].real for pr in plans}
    prof_err = (torch.linalg.norm(prof["mixed"] - prof["fp64"]) / torch.linalg.norm(prof["fp64"])).item()
    print(f"1000 steps: max energy rel err {worst:.2e}, mean-profile rel err {prof_err:.2e}")
    assert prof_err < 1e-6, prof_err
