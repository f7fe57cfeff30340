"""Generate the golden fixtures in tests/golden/*.npz from the reference itself.

Runs the unmodified reference package (dakling/jax-spectral-dns, read from
/root/reference) in FP64 on NumPy through the stand-in `jax` in
tests/golden/jax_shim, on seeded inputs built with the product's own seed
helper (jax_spectral_dns/seeds.py, loaded by file path so the reference's
package of the same name stays the one imported). Only this script reads
/root/reference; the fixtures it writes are small .npz files that travel with
the repository.

    python tests/golden/make_golden.py [case ...]

Each fixture stores the seeded input, the reference outputs after the listed
step counts, the energy history and the run parameters.
"""
from __future__ import annotations

import importlib.util
import math
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("JSD_REFERENCE", "/root/reference")

sys.path.insert(0, os.path.join(HERE, "jax_shim"))
sys.path.insert(1, REFERENCE)

_spec = importlib.util.spec_from_file_location(
    "jsd_seeds", os.path.join(REPO, "jax-spectral-dns_b200", "jax_spectral_dns", "seeds.py"))
seeds = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(seeds)

# the reference writes ./fields and ./plots; keep that out of the repository
os.chdir(tempfile.mkdtemp(prefix="jsd_golden_"))

import jax.numpy as jnp  # noqa: E402  (the shim)
from jax_spectral_dns.equation import Equation  # noqa: E402
from jax_spectral_dns.domain import PhysicalDomain  # noqa: E402
from jax_spectral_dns.field import FourierField, VectorField  # noqa: E402
from jax_spectral_dns.navier_stokes import NavierStokesVelVort  # noqa: E402
from jax_spectral_dns.navier_stokes_perturbation import NavierStokesVelVortPerturbation  # noqa: E402
from jax_spectral_dns.navier_stokes_perturbation_dual import NavierStokesVelVortPerturbationDual  # noqa: E402
from jax_spectral_dns.navier_stokes_perturbation_instationary import (  # noqa: E402
    NavierStokesVelVortPerturbationInstationary)

Equation.initialize()
Equation.verbosity_level = 0


def _domain(shape, lx, lz):
    return PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz), aliasing=3 / 2)


def _vf(dom, data):
    return VectorField.FromData(FourierField, dom, jnp.asarray(data), name="velocity_hat")


def _energy(dom, data):
    return float(_vf(dom, data).no_hat().energy())


def _run_forward(nse, dom, u0, dpdx0, n_steps, keep, energy_every=1):
    """Step the reference's perform_time_step by hand, recording states and E."""
    u = jnp.asarray(u0)
    dpdx = dpdx0
    states = {}
    dpdxs = [dpdx]
    energies = [_energy(dom, u)]
    for t in range(n_steps):
        u, dpdx = nse.perform_time_step(u, dpdx, t)
        dpdxs.append(float(dpdx))
        if (t + 1) % energy_every == 0:
            energies.append(_energy(dom, u))
        if (t + 1) in keep:
            states[t + 1] = np.asarray(u).copy()
    return states, np.array(energies), np.array(dpdxs)


def _save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, round(os.path.getsize(path) / 1024), "KiB", flush=True)


def case_lin_pert():
    """Linearised perturbation, pseudo-2D (Nz=4, Lz=2*pi*1e-3), Re=3000, dt=0.01,
    only kx=+-1, kz=0 populated, E0=1e-6 (the 9x65x5-mode pseudo-2D case)."""
    shape, lx, lz = (8, 65, 4), 2 * math.pi, 2 * math.pi * 1e-3
    re, dt, n = 3000.0, 0.01, 100
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (1, 0), 1e-6, seed=0)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=True)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep={1, 10, 100})
    _save("lin_pert_9x65x5", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt,
          u0=u0, u1=states[1], u10=states[10], u100=states[100], energy=en)


def case_lin_pert_gain():
    """Same pseudo-2D linearised case run to T=15 (1500 steps): energy every
    10 steps and the final gain."""
    shape, lx, lz = (8, 65, 4), 2 * math.pi, 2 * math.pi * 1e-3
    re, dt, n = 3000.0, 0.01, 1500
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (1, 0), 1e-6, seed=0)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=True)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep={n}, energy_every=10)
    _save("lin_pert_gain_9x65x5", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt,
          n_steps=n, energy_every10=en, u_final=states[n])


def case_nonlin_pert():
    """Nonlinear perturbation about Poiseuille flow, Re=5000, Lx=2pi, Lz=pi,
    9x33x9 modes with every mode populated (exercises the max-mode handling),
    E0=1e-3, dt=0.005."""
    shape, lx, lz = (8, 33, 8), 2 * math.pi, math.pi
    re, dt, n = 5000.0, 0.005, 20
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-3, seed=1)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=False)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep={1, 20})
    _save("nonlin_pert_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt,
          u0=u0, u1=states[1], u20=states[20], energy=en)


def case_nonlin_pert_odd():
    """Nonlinear perturbation on an uneven box: 5x24x13 modes (even Ny),
    Re=2000, Lx=3, Lz=5, E0=1e-2, dt=0.01."""
    shape, lx, lz = (4, 24, 12), 3.0, 5.0
    re, dt, n = 2000.0, 0.01, 5
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (2, 6), 1e-2, seed=2)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=False)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep={1, 5})
    _save("nonlin_pert_5x24x13", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt,
          u0=u0, u1=states[1], u5=states[5], energy=en)


def case_ns_cmf():
    """Full Navier-Stokes, constant mass flux, Re_tau=180, box 4pi x 2 x 4pi/3,
    9x33x9 modes, Reichardt mean profile + 10% perturbation, dt=0.002."""
    shape, lx, lz = (8, 33, 8), 4 * math.pi, 4 * math.pi / 3
    re_tau, dt, n = 180.0, 0.002, 10
    dom = _domain(shape, lx, lz)
    u0 = seeds.turbulent_channel_hat(shape, (lx, lz), re_tau, (4, 4), seed=3)
    nse = NavierStokesVelVort(_vf(dom, u0), Re_tau=re_tau, dt=dt, end_time=n * dt, constant_mass_flux=True)
    nse.activate_jit()
    dpdx0 = float(nse.dPdx)
    flow_rate = float(nse.flow_rate)
    states, en, dps = _run_forward(nse, dom, u0, dpdx0, n, keep={1, 10})
    _save("ns_cmf_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), re_tau=re_tau, dt=dt,
          u0=u0, u1=states[1], u10=states[10], energy=en, dpdx=dps, flow_rate=flow_rate)


def case_ns_cpg():
    """Full Navier-Stokes with a constant pressure gradient dPdx=-1,
    Re_tau=180, same box and seed family as the constant-mass-flux case."""
    shape, lx, lz = (8, 33, 8), 4 * math.pi, 4 * math.pi / 3
    re_tau, dt, n = 180.0, 0.002, 10
    dom = _domain(shape, lx, lz)
    u0 = seeds.turbulent_channel_hat(shape, (lx, lz), re_tau, (4, 4), seed=4)
    nse = NavierStokesVelVort(_vf(dom, u0), Re_tau=re_tau, dt=dt, end_time=n * dt, constant_mass_flux=False)
    nse.activate_jit()
    states, en, dps = _run_forward(nse, dom, u0, -1.0, n, keep={1, 10})
    _save("ns_cpg_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), re_tau=re_tau, dt=dt,
          u0=u0, u1=states[1], u10=states[10], energy=en, dpdx=dps)


def _dual_case(name, shape, lx, lz, re, dt, n, kmax, e0, seed, linearise):
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), kmax, e0, seed=seed)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=linearise)
    nse.activate_jit()
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse, checkpointing=False)
    t0 = time.time()
    grad = np.asarray(dual.get_grad()).copy()
    gain = float(dual.gain)
    uT = np.asarray(nse.get_latest_field("velocity_hat").get_data()).copy()
    print(name, "dual seconds", round(time.time() - t0, 1), "gain", gain, flush=True)
    _save(name, shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n,
          u0=u0, uT=uT, grad=grad, gain=gain)


def case_dual_lin():
    """Reference continuous-adjoint gradient, linearised, 5x33x5 pseudo-2D,
    Re=3000, T=0.2 (20 steps)."""
    _dual_case("dual_lin_5x33x5", (4, 33, 4), 2 * math.pi, 2 * math.pi * 1e-3, 3000.0, 0.01, 20,
               (1, 0), 1e-6, 5, True)


def case_dual_nonlin():
    """Reference continuous-adjoint gradient, nonlinear, 9x33x9, Re=3000,
    Lx=2pi, Lz=pi, E0=1e-4, T=0.05 (5 steps)."""
    _dual_case("dual_nonlin_9x33x9", (8, 33, 8), 2 * math.pi, math.pi, 3000.0, 0.01, 5,
               (4, 4), 1e-4, 6, False)


def case_instationary():
    """Perturbation about the accelerating wall-driven base flow of
    NavierStokesVelVortPerturbationInstationary (kappa = 1.5, n_max = 30,
    coupling_term off, base re-evaluated every step), Re=2000, 9x33x9 modes,
    E0=1e-3, dt=0.01, 12 steps."""
    shape, lx, lz = (8, 33, 8), 2 * math.pi, math.pi
    re, dt, n = 2000.0, 0.01, 12
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-3, seed=7)
    nse = NavierStokesVelVortPerturbationInstationary(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, kappa=1.5,
                                                      accelerate=True, n_max=30)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep={1, n})
    _save("instationary_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n,
          kappa=1.5, n_max=30, u0=u0, u1=states[1], un=states[n], energy=en)


def case_coupling_off():
    """Nonlinear perturbation about Poiseuille flow with coupling_term=False
    and linearised for the first half of the run (linearise_switch = 0.5),
    Re=3000, 9x33x9 modes, E0=1e-3, dt=0.01, 10 steps."""
    shape, lx, lz = (8, 33, 8), 2 * math.pi, math.pi
    re, dt, n = 3000.0, 0.01, 10
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-3, seed=8)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, coupling_term=False,
                                          linearise_switch=0.5)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep={1, n})
    _save("coupling_off_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n,
          linearise_switch=0.5, u0=u0, u1=states[1], un=states[n], energy=en)


def case_cg_opt():
    """Reference ConjugateGradientDescentSolver, 5 iterations, linearised
    pseudo-2D 5x33x5, Re=3000, T=0.2 (20 steps): gain per iteration and the
    final initial field."""
    from jax_spectral_dns.gradient_descent_solver import ConjugateGradientDescentSolver

    shape, lx, lz = (4, 33, 4), 2 * math.pi, 2 * math.pi * 1e-3
    re, dt, n = 3000.0, 0.01, 20
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (1, 0), 1e-6, seed=7)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=True)
    nse.activate_jit()
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse, checkpointing=False)
    gains = []

    solver = ConjugateGradientDescentSolver(dual, max_iterations=5, step_size=1e-2)
    # the optimise() loop without its plotting post-processing (gradient_descent_solver.py:114-124)
    solver.initialise(True)
    solver.update_done(solver.i)
    while not solver.done:
        solver.update()
        gains.append(float(solver.value))
        solver.i += 1
        solver.update_done(solver.i)
    final = np.asarray(solver.current_guess.get_data()).copy()
    _save("cg_opt_5x33x5", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n,
          u0=u0, gains=np.array(gains), final_guess=final, final_value=float(solver.value))


def case_dual_modes():
    """Reference continuous-adjoint gradients for the objectives gain_3d,
    gain_no_00 and dissipation (..._dual.py:388-400, 904-990, 1065-1104):
    linearised, 9x33x9 modes, Re=3000, Lx=2pi, Lz=pi, E0=1e-6, |kx|,|kz| <= 4,
    dt=0.01, T=0.1. The dissipation objective only sees the (0, 0) mode (the
    x-z integral of the squared spectral gradients), which the seeded field
    leaves at zero, so its case adds a streamwise mean-flow perturbation
    1e-3 (1 - y^2) to make the value more than the transforms' round-off."""
    shape, lx, lz = (8, 33, 8), 2 * math.pi, math.pi
    re, dt, n = 3000.0, 0.01, 10
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-6, seed=12)
    u0_diss = u0.copy()
    u0_diss[0, 0, :, 0] += 1e-3 * (1.0 - seeds.cheb_points(u0.shape[2]) ** 2)
    out = {"dissipation_u0": u0_diss}
    for mode in ("gain_3d", "gain_no_00", "dissipation"):
        start = u0_diss if mode == "dissipation" else u0
        nse = NavierStokesVelVortPerturbation(_vf(dom, start), Re=re, dt=dt, end_time=n * dt, linearise=True)
        nse.activate_jit()
        dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(
            nse, checkpointing=False, optimisation_mode=mode)
        value = float(dual.get_objective_fun())
        grad = np.asarray(dual.get_grad()).copy()
        out[mode + "_value"] = value
        out[mode + "_grad"] = grad
        print(mode, value, flush=True)
    _save("dual_modes_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n, u0=u0,
          **out)


def _no_plots():
    """The solvers plot the gradient after successful steps; plotting is not
    part of the arithmetic, so the field plot methods are made no-ops here."""
    from jax_spectral_dns.field import Field, PhysicalField, VectorField as VF

    for cls in (Field, PhysicalField, VF):
        for nm in ("plot_3d", "plot_center", "plot", "plot_2d"):
            if hasattr(cls, nm):
                setattr(cls, nm, lambda *a, **k: None)


def case_solvers():
    """Reference solvers on the linearised pseudo-2D 5x33x5 problem (Re=3000,
    T=0.2, 20 steps, E0=1e-6): ConjugateGradientDescentSolver with the line
    search, 3 iterations; SteepestAdaptiveDescentSolver on the same problem
    with T = 2, initialisation and 2 updates (its trial problems are nonlinear
    perturbations)."""
    from jax_spectral_dns.gradient_descent_solver import (ConjugateGradientDescentSolver,
                                                          SteepestAdaptiveDescentSolver)

    _no_plots()
    shape, lx, lz = (4, 33, 4), 2 * math.pi, 2 * math.pi * 1e-3
    re, dt, n = 3000.0, 0.01, 20
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (1, 0), 1e-6, seed=7)
    res = {}
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=True)
    nse.activate_jit()
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse, checkpointing=False)
    solver = ConjugateGradientDescentSolver(dual, max_iterations=3, step_size=1e-2, use_linesearch=True)
    solver.initialise(True)
    ls_values, ls_steps = [], []
    for it in range(3):
        solver.update()
        ls_values.append(float(solver.value))
        ls_steps.append(float(solver.step_size))
        solver.i += 1
    res.update(ls_values=np.array(ls_values), ls_steps=np.array(ls_steps),
               ls_final=np.asarray(solver.current_guess.get_data()).copy())
    # the steepest solver re-chooses dt from the CFL number (about 0.2 here), so
    # it needs a horizon of several such steps: T = 2 (200 steps of 0.01 at first)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=10 * n * dt, linearise=True)
    nse.activate_jit()
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse, checkpointing=False)
    st = SteepestAdaptiveDescentSolver(dual, max_iterations=3, step_size=1e-2)
    st.initialise(True)
    sd_values, sd_steps, sd_dts = [float(st.value)], [float(st.step_size)], [float(st.dual_problem.forward_equation.get_dt())]
    for it in range(2):
        st.update()
        sd_values.append(float(st.value))
        sd_steps.append(float(st.step_size))
        sd_dts.append(float(st.dual_problem.forward_equation.get_dt()))
        st.i += 1
    res.update(sd_values=np.array(sd_values), sd_steps=np.array(sd_steps), sd_dts=np.array(sd_dts),
               sd_final=np.asarray(st.current_guess.get_data()).copy())
    print("line search", ls_values, ls_steps, "steepest", sd_values, sd_steps, sd_dts, flush=True)
    _save("solvers_5x33x5", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n, u0=u0, **res)


def case_lsc():
    """Reference LinearStabilityCalculation (n = 50): eigenvalues, leading
    eigenvectors, optimal gains and coefficients for three (Re, alpha, beta,
    T) cases, and the optimal initial field on the 5x50x5-mode box of the
    reference's run_transient_growth (examples.py:1274-1324)."""
    from jax_spectral_dns.linear_stability_calculation import LinearStabilityCalculation

    out = {}
    for tag, re, alpha, beta, t, modes in (("re3000", 3000.0, 1.0, 0.0, 15.0, 60),
                                           ("re600", 600.0, 1.0, 0.0, 2.0, 60),
                                           ("re1000b", 1000.0, 1.0, 1.0, 10.0, 40)):
        lsc = LinearStabilityCalculation(Re=re, alpha=alpha, beta=beta, n=50)
        evs, evecs = lsc.calculate_eigenvalues()
        s, coeffs = lsc.calculate_transient_growth_svd(t, modes, save=False)
        out[tag + "_params"] = np.array([re, alpha, beta, t, modes])
        out[tag + "_evs"] = np.asarray(evs)
        out[tag + "_evecs3"] = np.array(evecs[:3])
        out[tag + "_S"] = np.asarray(s)
        out[tag + "_coeffs"] = np.asarray(coeffs)
        if tag == "re3000":
            out[tag + "_gains_T"] = np.array([2.0, 5.0, 10.0])
            out[tag + "_gains"] = np.array([float(lsc.calculate_transient_growth_svd(tt, modes)[0][0] ** 2)
                                            for tt in (2.0, 5.0, 10.0)])
            dom = PhysicalDomain.create((4, 50, 4), (True, False, True),
                                        scale_factors=(2 * math.pi / alpha, 1.0, 1.0e-3), aliasing=3 / 2)
            u = lsc.calculate_transient_growth_initial_condition(dom, t, modes, recompute_full=True,
                                                                 save_final=False)
            out[tag + "_ic"] = np.array([np.asarray(u[i].data) for i in range(3)])
            out[tag + "_ic_energy"] = float(u.energy())
            out[tag + "_mode0_energy"] = float(lsc.velocity_field_single_mode(dom, 0, recompute_partial=True).energy())
    lsc = LinearStabilityCalculation(Re=5772.22, alpha=1.02056, n=50)
    out["neutral_evs"] = np.asarray(lsc.calculate_eigenvalues()[0][:5])
    _save("lsc_n50", **out)


def case_vort_yvel():
    """Reference NavierStokesVelVort.vort_yvel_to_vel and
    smooth_and_enforce_bc_vel_y (navier_stokes.py:1027-1203) on seeded
    spectral omega_y and v (9x33x9 modes, box 2pi x 2 x pi), in 3-D and with
    two_d=True."""
    shape, lx, lz = (8, 33, 8), 2 * math.pi, math.pi
    dom = _domain(shape, lx, lz)
    rng = np.random.default_rng(12)
    mx, ny, mz = 9, 33, 9
    vort = rng.standard_normal((mx, ny, mz)) + 1j * rng.standard_normal((mx, ny, mz))
    vel_y = rng.standard_normal((mx, ny, mz)) + 1j * rng.standard_normal((mx, ny, mz))
    ux00 = rng.standard_normal(ny)
    uz00 = rng.standard_normal(ny)
    out3 = np.asarray(NavierStokesVelVort.vort_yvel_to_vel(dom, jnp.asarray(vort), jnp.asarray(vel_y),
                                                           jnp.asarray(ux00), jnp.asarray(uz00)))
    out2 = np.asarray(NavierStokesVelVort.vort_yvel_to_vel(dom, None, jnp.asarray(vel_y), jnp.asarray(ux00),
                                                           None, two_d=True))
    vs = rng.standard_normal(ny)
    sm = np.asarray(NavierStokesVelVort.smooth_and_enforce_bc_vel_y(dom, jnp.asarray(vs)))
    sm10 = np.asarray(NavierStokesVelVort.smooth_and_enforce_bc_vel_y(dom, jnp.asarray(vs), M=10))
    _save("vort_yvel_9x33x9", shape=np.array(shape), lengths=np.array([lx, lz]), vort=vort, vel_y=vel_y,
          ux00=ux00, uz00=uz00, out3=out3, out2=out2, slice_in=vs, slice_out=sm, slice_out_m10=sm10)


SAMPLE_SEED, N_SAMPLES = 1234, 4096


def _sample(a):
    """A fixed seeded sample of a large state (the fixture keeps it, its norm
    and the energy history instead of the whole array)."""
    flat = np.asarray(a).ravel()
    idx = np.sort(np.random.default_rng(SAMPLE_SEED).choice(flat.size, N_SAMPLES, replace=False))
    return idx, flat[idx]


def case_config1():
    """Nonlinear perturbation at the size of BASELINE config 1: 49x65x49 modes
    (48x65x48), Re=5000, Lx=2pi, Lz=pi, dt=0.005, E0=1e-3, |kx|,|kz| <= 8,
    seed 0; 100 steps. States after 1, 10, 50 and 100 steps kept as seeded
    samples plus norms, with the energy after every step."""
    shape, lx, lz = (48, 65, 48), 2 * math.pi, math.pi
    re, dt, n = 5000.0, 0.005, 100
    keep = (1, 10, 50, 100)
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-3, seed=0)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=False)
    nse.activate_jit()
    states, en, _ = _run_forward(nse, dom, u0, 0.0, n, keep=set(keep))
    idx, s0 = _sample(u0)
    extra = {}
    for k in keep:
        _, sk = _sample(states[k])
        extra[f"u{k}_sample"] = sk
        extra[f"u{k}_norm"] = np.linalg.norm(states[k])
    _save("config1_49x65x49", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n,
          kmax=np.array([8, 8]), e0=1e-3, seed=0, idx=idx, u0_sample=s0, u0_norm=np.linalg.norm(u0),
          kept_steps=np.array(keep), energy=en, **extra)


def case_config2_dual():
    """Reference dual-solver gradient at the size of BASELINE config 2:
    33x65x33 modes (32x65x32), Re=3000, Lx=2pi, Lz=pi, dt=0.01, T=0.5
    (50 steps), linearised, E0=1e-6, |kx|,|kz| <= 8, seed 2. Gradient kept as a
    seeded sample plus its norm."""
    shape, lx, lz = (32, 65, 32), 2 * math.pi, math.pi
    re, dt, n = 3000.0, 0.01, 50
    dom = _domain(shape, lx, lz)
    u0 = seeds.seeded_velocity_hat(shape, (lx, lz), (8, 8), 1e-6, seed=2)
    nse = NavierStokesVelVortPerturbation(_vf(dom, u0), Re=re, dt=dt, end_time=n * dt, linearise=True)
    nse.activate_jit()
    dual = NavierStokesVelVortPerturbationDual.FromNavierStokesVelVortPerturbation(nse, checkpointing=False)
    grad = np.asarray(dual.get_grad()).copy()
    gain = float(dual.gain)
    idx, s0 = _sample(u0)
    _, sg = _sample(grad)
    _save("config2_dual_33x65x33", shape=np.array(shape), lengths=np.array([lx, lz]), re=re, dt=dt, n_steps=n,
          kmax=np.array([8, 8]), e0=1e-6, seed=2, idx=idx, u0_sample=s0, grad_sample=sg,
          u0_norm=np.linalg.norm(u0), grad_norm=np.linalg.norm(grad), gain=gain)


def case_config4():
    """The benchmark workload itself: NS with constant mass flux, Re_tau = 180,
    box 4pi x 2 x 4pi/3, 129x129x129 modes (128x129x128), dt = 0.002, the
    seeded Reichardt-plus-perturbation field of bench.py (|kx|, |kz| <= 16,
    seed 0); 3 steps. States after 1 and 3 steps kept as seeded samples plus
    norms, with dPdx and the energy after every step."""
    shape, lx, lz = (128, 129, 128), 4 * math.pi, 4 * math.pi / 3
    re_tau, dt, n = 180.0, 0.002, 3
    dom = _domain(shape, lx, lz)
    u0 = seeds.turbulent_channel_hat(shape, (lx, lz), re_tau, (16, 16), seed=0)
    nse = NavierStokesVelVort(_vf(dom, u0), Re_tau=re_tau, dt=dt, end_time=n * dt, constant_mass_flux=True)
    nse.activate_jit()
    dpdx0 = float(nse.dPdx)
    flow_rate = float(nse.flow_rate)
    t0 = time.time()
    states, en, dps = _run_forward(nse, dom, u0, dpdx0, n, keep={1, n})
    print("config4 seconds per step", round((time.time() - t0) / n, 1), flush=True)
    idx, s0 = _sample(u0)
    _, s1 = _sample(states[1])
    _, s3 = _sample(states[n])
    _save("config4_129x129x129", shape=np.array(shape), lengths=np.array([lx, lz]), re_tau=re_tau, dt=dt,
          n_steps=n, kmax=np.array([16, 16]), seed=0, idx=idx, u0_sample=s0, u1_sample=s1, u3_sample=s3,
          u0_norm=np.linalg.norm(u0), u1_norm=np.linalg.norm(states[1]), u3_norm=np.linalg.norm(states[n]),
          energy=en, dpdx=dps, flow_rate=flow_rate)


CASES = {
    "config4": case_config4,
    "config1": case_config1,
    "config2_dual": case_config2_dual,
    "vort_yvel": case_vort_yvel,
    "lsc": case_lsc,
    "lin_pert": case_lin_pert,
    "lin_pert_gain": case_lin_pert_gain,
    "nonlin_pert": case_nonlin_pert,
    "nonlin_pert_odd": case_nonlin_pert_odd,
    "ns_cmf": case_ns_cmf,
    "ns_cpg": case_ns_cpg,
    "dual_lin": case_dual_lin,
    "dual_nonlin": case_dual_nonlin,
    "cg_opt": case_cg_opt,
    "dual_modes": case_dual_modes,
    "solvers": case_solvers,
    "instationary": case_instationary,
    "coupling_off": case_coupling_off,
}

if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        t = time.time()
        CASES[nm]()
        print(nm, "done in", round(time.time() - t, 1), "s", flush=True)
