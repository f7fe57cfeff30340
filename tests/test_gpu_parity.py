"""Parity of the native B200 step (through the C ABI) with the reference.

Small cases compare with the golden fixtures the unmodified reference produced;
medium and full-size cases compare with the CPU oracle on the same seeded
inputs, or check size-independent properties (linearity, determinism).
Tolerance: relative L2 <= 1e-10 on the spectral state (the FP64 parity bar).
"""
import numpy as np
import pytest
import torch

import jsd_oracle as O
from conftest import golden, rel
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat, turbulent_channel_hat

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _pert_plan(shape, lengths, re, dt, linearise, kind=1, dt_explicit=None):
    modes, phys = mode_counts(tuple(shape))
    return StepPlan(modes, phys, *lengths, kind, float(re), float(dt), dt_explicit=dt_explicit,
                    linearise=linearise, base_u=1 - cheb_points(modes[1]) ** 2)


def _run(plan, u0, n, dpdx0=0.0, keep=()):
    st = to_device_layout(u0)
    dp = torch.tensor([dpdx0], dtype=torch.float64, device="cuda")
    out = {}
    for t in range(n):
        plan.step(st, dp, t, 1)
        if t + 1 in keep:
            out[t + 1] = to_reference_layout(st).cpu().numpy()
    return st, dp, out


def test_linear_perturbation_100_steps(cuda):
    d = golden("lin_pert_9x65x5")
    p = _pert_plan(d["shape"], d["lengths"], d["re"], d["dt"], True)
    st, _, out = _run(p, d["u0"], 100, keep={1, 10, 100})
    for k in (1, 10, 100):
        assert rel(out[k], d["u%d" % k]) < TOL
    # energy history through the native reduction
    assert abs(p.energy(st).item() / d["energy"][100] - 1) < TOL


def test_linear_perturbation_gain_T15(cuda):
    """1500 steps to T = 15: the transient-growth gain and E(t) every 10 steps."""
    d = golden("lin_pert_gain_9x65x5")
    g0 = golden("lin_pert_9x65x5")
    p = _pert_plan(d["shape"], d["lengths"], d["re"], d["dt"], True)
    st = to_device_layout(g0["u0"])
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    en = [p.energy(st).item()]
    for k in range(150):
        p.step(st, dp, 10 * k, 10)
        en.append(p.energy(st).item())
    en = np.array(en)
    assert np.abs(en / d["energy_every10"] - 1).max() < TOL
    assert rel(to_reference_layout(st).cpu().numpy(), d["u_final"]) < TOL


@pytest.mark.parametrize("name,steps", [("nonlin_pert_9x33x9", 20), ("nonlin_pert_5x24x13", 5)])
def test_nonlinear_perturbation(cuda, name, steps):
    d = golden(name)
    p = _pert_plan(d["shape"], d["lengths"], d["re"], d["dt"], False)
    _, _, out = _run(p, d["u0"], steps, keep={1, steps})
    assert rel(out[1], d["u1"]) < TOL
    assert rel(out[steps], d["u%d" % steps]) < TOL


@pytest.mark.parametrize("name,cmf", [("ns_cmf_9x33x9", True), ("ns_cpg_9x33x9", False)])
def test_navier_stokes(cuda, name, cmf):
    d = golden(name)
    modes, phys = mode_counts(tuple(d["shape"]))
    probe = StepPlan(modes, phys, *d["lengths"], 0, float(d["re_tau"]), float(d["dt"]))
    q0 = probe.flow_rate(to_device_layout(d["u0"])[0]).item()
    if cmf:
        assert abs(q0 / float(d["flow_rate"]) - 1) < 1e-13
    p = StepPlan(modes, phys, *d["lengths"], 0, float(d["re_tau"]), float(d["dt"]), constant_mass_flux=cmf,
                 flow_rate_target=q0)
    _, dp, out = _run(p, d["u0"], 10, float(d["dpdx"][0]), keep={1, 10})
    assert rel(out[1], d["u1"]) < TOL
    assert rel(out[10], d["u10"]) < TOL
    assert abs(dp.item() - d["dpdx"][-1]) < 1e-8 * max(1.0, abs(d["dpdx"][-1]))


def test_dual_linear_gradient(cuda):
    d = golden("dual_lin_5x33x5")
    n, dt = int(d["n_steps"]), float(d["dt"])
    fwd = _pert_plan(d["shape"], d["lengths"], d["re"], dt, True)
    st, _, _ = _run(fwd, d["u0"], n)
    e0 = fwd.energy(to_device_layout(d["u0"])).item()
    gain = fwd.energy(st).item() / e0
    dual = _pert_plan(d["shape"], d["lengths"], d["re"], dt, True, kind=2, dt_explicit=-dt)
    v = (-st).contiguous()
    dual.step(v, torch.zeros(1, dtype=torch.float64, device="cuda"), 0, n)
    grad = (d["u0"] - to_reference_layout(v).cpu().numpy()) / e0
    assert rel(grad, d["grad"]) < TOL
    assert abs(gain / float(d["gain"]) - 1) < TOL


def test_nonlinear_perturbation_49x65x49_vs_oracle(cuda):
    """The 48x65x48-mode configuration (Re = 5000, Lx = 2 pi, Lz = pi), |k| <= 8
    seeded, 3 steps against the oracle on the same input."""
    shape, lx, lz, re, dt = (48, 65, 48), 2 * np.pi, np.pi, 5000.0, 0.005
    u0 = seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-3, seed=21)
    p = _pert_plan(shape, (lx, lz), re, dt, False)
    _, _, out = _run(p, u0, 3, keep={3})
    want, _, _ = O.run(O.make_stepper("perturbation", shape, lx, lz, re, dt, linearise=False), u0, 3)
    assert rel(out[3], want) < TOL


def test_channel_128x129x128_one_step_vs_oracle(cuda):
    """Full-size turbulent-channel configuration: one constant-mass-flux step
    from the seeded Reichardt field against the oracle (about a minute of CPU)."""
    shape, lx, lz, re_tau, dt = (128, 129, 128), 4 * np.pi, 4 * np.pi / 3, 180.0, 0.002
    u0 = turbulent_channel_hat(shape, (lx, lz), re_tau, (16, 16), seed=0)
    modes, phys = mode_counts(shape)
    probe = StepPlan(modes, phys, lx, lz, 0, re_tau, dt)
    q0 = probe.flow_rate(to_device_layout(u0)[0]).item()
    p = StepPlan(modes, phys, lx, lz, 0, re_tau, dt, constant_mass_flux=True, flow_rate_target=q0)
    dpdx0 = -q0 * 3 / 2 / re_tau
    _, dp, out = _run(p, u0, 1, dpdx0, keep={1})
    g = O.Grid(shape, lx, lz)
    st = O.Stepper(g, re_tau, dt, kind="ns", constant_mass_flux=True, flow_rate_target=g.flow_rate(u0[0]))
    want, dp_want = st.rk_step(u0, dpdx0, 0)
    assert rel(out[1], want) < TOL
    assert abs(dp.item() - dp_want) < 1e-8 * max(1.0, abs(dp_want))


def test_linearised_step_is_linear_at_full_size(cuda):
    """Size-independent property at 129 x 129 x 129 modes: the linearised
    perturbation step is real-linear, S(a u + b w) = a S(u) + b S(w)."""
    shape, lx, lz = (128, 129, 128), 2 * np.pi, np.pi
    u = seeded_velocity_hat(shape, (lx, lz), (16, 16), 1e-4, seed=1)
    w = seeded_velocity_hat(shape, (lx, lz), (16, 16), 1e-4, seed=2)
    p = _pert_plan(shape, (lx, lz), 3000.0, 0.01, True)
    su, _, _ = _run(p, u, 2)
    sw, _, _ = _run(p, w, 2)
    sc, _, _ = _run(p, 0.3 * u - 1.7 * w, 2)
    comb = 0.3 * su - 1.7 * sw
    assert (torch.linalg.norm(sc - comb) / torch.linalg.norm(comb)).item() < 1e-12


def test_deterministic_and_finite_full_size(cuda):
    shape, lx, lz, re_tau, dt = (128, 129, 128), 4 * np.pi, 4 * np.pi / 3, 180.0, 0.002
    u0 = turbulent_channel_hat(shape, (lx, lz), re_tau, (16, 16), seed=0)
    modes, phys = mode_counts(shape)
    p = StepPlan(modes, phys, lx, lz, 0, re_tau, dt)
    a, _, _ = _run(p, u0, 3, -1.0)
    b, _, _ = _run(p, u0, 3, -1.0)
    assert torch.equal(a, b)
    assert bool(torch.isfinite(torch.view_as_real(a)).all())


def test_dual_nonlinear_gradient(cuda):
    """Nonlinear adjoint: the forward trajectory is registered with the plan
    (jsd_set_history) and dual step t uses u(T - t) for all three stages."""
    d = golden("dual_nonlin_9x33x9")
    n, dt = int(d["n_steps"]), float(d["dt"])
    fwd = _pert_plan(d["shape"], d["lengths"], d["re"], dt, False)
    st = to_device_layout(d["u0"])
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    traj = torch.empty((n + 1,) + tuple(st.shape), dtype=st.dtype, device=st.device)
    traj[0].copy_(st)
    for t in range(n):
        fwd.step(st, dp, t, 1)
        traj[t + 1].copy_(st)
    e0 = fwd.energy(traj[0]).item()
    dual = _pert_plan(d["shape"], d["lengths"], d["re"], dt, False, kind=2, dt_explicit=-dt)
    dual.set_history(traj)
    v = (-st).contiguous()
    dual.step(v, dp, 0, n)
    grad = (d["u0"] - to_reference_layout(v).cpu().numpy()) / e0
    assert rel(grad, d["grad"]) < TOL
    assert rel(to_reference_layout(st).cpu().numpy(), d["uT"]) < TOL
