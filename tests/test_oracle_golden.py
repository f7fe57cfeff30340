"""The CPU oracle against outputs of the unmodified reference (golden fixtures).

These pin the oracle: each fixture was produced by the reference package
itself (tests/golden/make_golden.py), so agreement to ~1e-12 here means the
oracle restates the reference's arithmetic, quirks included.
"""
import os

import numpy as np
import pytest

import jsd_oracle as O
from conftest import golden, rel


def _pert(d, linearise):
    return O.make_stepper("perturbation", tuple(d["shape"]), *d["lengths"], float(d["re"]), float(d["dt"]),
                          linearise=linearise)


def test_linearised_perturbation_pseudo2d():
    d = golden("lin_pert_9x65x5")
    st = _pert(d, True)
    u = d["u0"]
    for t in range(10):
        u, _ = st.rk_step(u, 0.0, t)
        if t == 0:
            assert rel(u, d["u1"]) < 1e-12
    assert rel(u, d["u10"]) < 1e-12
    assert abs(st.g.energy(u) / d["energy"][10] - 1) < 1e-12


@pytest.mark.parametrize("name,steps", [("nonlin_pert_9x33x9", 20), ("nonlin_pert_5x24x13", 5)])
def test_nonlinear_perturbation(name, steps):
    d = golden(name)
    st = _pert(d, False)
    u, _, _ = O.run(st, d["u0"], steps)
    assert rel(u, d["u%d" % steps]) < 1e-12


@pytest.mark.parametrize("name,cmf", [("ns_cmf_9x33x9", True), ("ns_cpg_9x33x9", False)])
def test_navier_stokes(name, cmf):
    d = golden(name)
    g = O.Grid(tuple(d["shape"]), *d["lengths"])
    q0 = g.flow_rate(d["u0"][0])
    if cmf:
        assert abs(q0 / float(d["flow_rate"]) - 1) < 1e-13
    st = O.Stepper(g, float(d["re_tau"]), float(d["dt"]), kind="ns", constant_mass_flux=cmf, flow_rate_target=q0)
    u, dp, _ = O.run(st, d["u0"], 10, dpdx=float(d["dpdx"][0]))
    assert rel(u, d["u10"]) < 1e-12
    assert abs(dp - d["dpdx"][-1]) < 1e-9 * max(1.0, abs(dp))


@pytest.mark.parametrize("name,lin", [("dual_lin_5x33x5", True), ("dual_nonlin_9x33x9", False)])
def test_dual_gradient(name, lin):
    d = golden(name)
    grad, gain, _, uT = O.dual_gradient(tuple(d["shape"]), *d["lengths"], float(d["re"]), float(d["dt"]),
                                        int(d["n_steps"]), d["u0"], lin)
    assert rel(grad, d["grad"]) < 1e-12
    assert rel(uT, d["uT"]) < 1e-12
    assert abs(gain / float(d["gain"]) - 1) < 1e-13


def test_dissipation_objective():
    """The dual's dissipation objective (navier_stokes_perturbation_dual.py:
    904-990, 1089-1120): the source from the forward history in every dual
    step, composed with the reference's indexing (navier_stokes.py:1461-1491,
    1697-1703), and the time-averaged value."""
    d = golden("dual_modes_9x33x9")
    grad, value, _ = O.dissipation_gradient(tuple(d["shape"]), *d["lengths"], float(d["re"]), float(d["dt"]),
                                            int(d["n_steps"]), d["dissipation_u0"], True)
    assert rel(grad, d["dissipation_grad"]) < 1e-12
    assert abs(value / float(d["dissipation_value"]) - 1) < 1e-10


def test_transient_growth_energy_history():
    """E(t) over the first 100 steps of the pseudo-2D linear case."""
    d = golden("lin_pert_9x65x5")
    e = d["energy"]
    assert e.shape == (101,)
    assert np.all(np.isfinite(e)) and e[0] > 0
    assert abs(e[0] / 1e-6 - 1) < 1e-10  # seeded at E0 = 1e-6


def test_instationary_base_flow():
    """Wall-driven accelerating base re-evaluated every step, coupling_term
    off (NavierStokesVelVortPerturbationInstationary)."""
    d = golden("instationary_9x33x9")
    n, dt, re = int(d["n_steps"]), float(d["dt"]), float(d["re"])
    st = _pert(d, False)
    st.coupling_term = False
    st.base_fn = lambda t: O.instationary_base_hat(st.g, t * dt, re, float(d["kappa"]), True, int(d["n_max"]))
    u, _, _ = O.run(st, d["u0"], n)
    assert rel(u, d["un"]) < 1e-12


def test_coupling_off_with_linearise_switch():
    d = golden("coupling_off_9x33x9")
    n = int(d["n_steps"])
    st = _pert(d, False)
    st.coupling_term = False
    st.linearise = lambda t: t < n * float(d["linearise_switch"])
    u1, _, _ = O.run(st, d["u0"], 1)
    assert rel(u1, d["u1"]) < 1e-12
    u, _, _ = O.run(st, d["u0"], n)
    assert rel(u, d["un"]) < 1e-12


def test_oracle_at_config1_size():
    """The oracle's first step at 49x65x49 modes (Re = 5000, dt = 0.005, every
    |kx|, |kz| <= 8 populated) against the reference's, through the fixture's
    seeded sample and norm (tests/golden/config1_49x65x49.npz)."""
    from jax_spectral_dns.seeds import seeded_velocity_hat

    d = golden("config1_49x65x49")
    shape, (lx, lz) = tuple(int(x) for x in d["shape"]), d["lengths"]
    u0 = seeded_velocity_hat(shape, (lx, lz), tuple(int(k) for k in d["kmax"]), float(d["e0"]), seed=int(d["seed"]))
    st = O.make_stepper("perturbation", shape, lx, lz, float(d["re"]), float(d["dt"]), linearise=False)
    u1, _, _ = O.run(st, u0, 1)
    f = u1.ravel()
    assert np.linalg.norm(f[d["idx"]] - d["u1_sample"]) < 1e-12 * np.linalg.norm(d["u1_sample"])
    assert abs(np.linalg.norm(u1) / float(d["u1_norm"]) - 1) < 1e-12


@pytest.mark.skipif(not os.environ.get("JSD_SLOW_TESTS"), reason="about 3 minutes on CPU; set JSD_SLOW_TESTS=1")
def test_oracle_dual_gradient_at_config2_size():
    """The oracle's dual gradient at 33x65x33 modes (Re = 3000, T = 0.5,
    linearised) against the reference dual solver's, through the fixture's
    seeded sample and norm (tests/golden/config2_dual_33x65x33.npz)."""
    from jax_spectral_dns.seeds import seeded_velocity_hat

    d = golden("config2_dual_33x65x33")
    shape, (lx, lz) = tuple(int(x) for x in d["shape"]), d["lengths"]
    u0 = seeded_velocity_hat(shape, (lx, lz), tuple(int(k) for k in d["kmax"]), float(d["e0"]), seed=int(d["seed"]))
    g, gain, _, _ = O.dual_gradient(shape, lx, lz, float(d["re"]), float(d["dt"]), int(d["n_steps"]), u0, True)
    f = g.ravel()
    assert np.linalg.norm(f[d["idx"]] - d["grad_sample"]) < 1e-12 * np.linalg.norm(d["grad_sample"])
    assert abs(gain / float(d["gain"]) - 1) < 1e-12
