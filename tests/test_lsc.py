"""LinearStabilityCalculation against the reference's own outputs
(tests/golden/lsc_n50.npz, written by make_golden.py case ``lsc``).

Eigenvector phases, and the phase of the optimal singular vector, are fixed
by LAPACK's internal choices; quantities that depend on them are compared up
to those phases (per eigenvector, and one global phase for the optimal
initial field: a shift in x)."""
import math
import os

import numpy as np
import pytest
import torch

from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.linear_stability_calculation import (LinearStabilityCalculation, basis_matrix,
                                                          gram_matrix)

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "lsc_n50.npz"))
CASES = ("re3000", "re600", "re1000b")


def _lsc(tag):
    re, alpha, beta, t, modes = GOLDEN[tag + "_params"]
    return LinearStabilityCalculation(Re=re, alpha=alpha, beta=beta, n=50), float(t), int(modes)


def _phase_aligned(a, b):
    """b times the unit complex factor that best aligns it with a."""
    z = np.vdot(b, a)
    return b * (z / abs(z))


@pytest.mark.parametrize("tag", CASES)
def test_eigenvalues_match_reference(tag):
    lsc, _, _ = _lsc(tag)
    evs, evecs = lsc.calculate_eigenvalues()
    ref = GOLDEN[tag + "_evs"]
    assert evs.shape == ref.shape
    lead = slice(0, 60)
    np.testing.assert_allclose(evs[lead], ref[lead], rtol=0, atol=1e-10 * np.abs(ref[lead]).max())
    for j in range(3):
        a, b = GOLDEN[tag + "_evecs3"][j], evecs[j]
        assert np.linalg.norm(_phase_aligned(a, b) - a) < 1e-9 * np.linalg.norm(a)


@pytest.mark.parametrize("tag", CASES)
def test_optimal_gain_matches_reference(tag):
    lsc, t, modes = _lsc(tag)
    s, coeffs = lsc.calculate_transient_growth_svd(t, modes)
    ref = GOLDEN[tag + "_S"]
    # the Gram matrix of nearly parallel non-normal modes is ill-conditioned:
    # round-off in C (summation order) moves every singular value by up to
    # ~1e-9 S_1 in the reference itself, so the bound is absolute in S_1
    np.testing.assert_allclose(s, ref, rtol=0, atol=1e-8 * ref[0])
    assert abs(s[0] ** 2 / ref[0] ** 2 - 1) < 1e-8


def test_gain_curve_batched_svd():
    lsc, _, modes = _lsc("re3000")
    ts = GOLDEN["re3000_gains_T"]
    g = lsc.transient_growth_gains(ts, modes)
    np.testing.assert_allclose(g, GOLDEN["re3000_gains"], rtol=1e-8)
    g_cpu = lsc.transient_growth_gains(ts, modes, device=torch.device("cpu"))
    np.testing.assert_allclose(g, g_cpu, rtol=1e-12)


def test_optimal_initial_condition_matches_reference():
    lsc, t, modes = _lsc("re3000")
    dom = PhysicalDomain.create((4, 50, 4), (True, False, True), scale_factors=(2 * math.pi, 1.0, 1.0e-3))
    u = lsc.calculate_transient_growth_initial_condition(dom, t, modes, recompute_full=True)
    ours = np.array([u[i].data.cpu().numpy() for i in range(3)])
    ref = GOLDEN["re3000_ic"]
    assert ours.shape == ref.shape
    # Re(c f(y) e^{i x}): compare the kx = 1 Fourier coefficient up to one
    # global phase. The coefficients F^-1 v_1 pass through the Cholesky factor
    # of the Gram matrix C, whose condition number is ~9e8 here: round-off in
    # C alone moves the field by up to cond(C) eps ~ 1e-7
    a = np.fft.fft(ref, axis=1)[:, 1].ravel()
    b = np.fft.fft(ours, axis=1)[:, 1].ravel()
    assert np.linalg.norm(_phase_aligned(a, b) - a) < 1e-7 * np.linalg.norm(a)
    assert abs(u.energy() / float(GOLDEN["re3000_ic_energy"]) - 1) < 1e-7
    e_max = lsc.calculate_transient_growth_max_energy(t, modes)
    assert abs(e_max / GOLDEN["re3000_S"][0] ** 2 - 1) < 1e-8
    mode0 = lsc.velocity_field_single_mode(dom, 0)
    assert abs(mode0.energy() / float(GOLDEN["re3000_mode0_energy"]) - 1) < 1e-9


def test_neutral_curve_point():
    """The reference's test_linear_stability (tests/test_project.py:1225-1236):
    at Re = 5772.22, alpha = 1.02056 the leading eigenvalue is neutral."""
    lsc = LinearStabilityCalculation(Re=5772.22, alpha=1.02056, n=50)
    evs, _ = lsc.calculate_eigenvalues()
    assert -1e-8 <= evs[0].real <= 0.0
    np.testing.assert_allclose(evs[:5], GOLDEN["neutral_evs"], rtol=0, atol=1e-10)


def test_gram_integrals_exact():
    """Exact Chebyshev Gram integrals equal high-order Gauss-Legendre quadrature."""
    x, w = np.polynomial.legendre.leggauss(80)
    for kind in ("a", "s", "full"):
        m = basis_matrix(kind, 12, x)
        np.testing.assert_allclose(gram_matrix(kind, 12), (m * w[:, None]).T @ m, rtol=0, atol=1e-13)


def test_optimal_growth_through_oracle_step():
    """The reference's transient-growth check (tests/test_project.py:1489-1503,
    run_transient_growth, examples.py:1274-1413) at Re = 600, T = 2 with the
    oracle's linearised step: the energy gain of the optimal initial field
    after 200 steps equals the predicted optimal gain. The reference accepts
    8e-4; the two agree to ~2e-7 (time-discretisation error)."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    import jsd_oracle as O

    re, t = 600.0, 2.0
    dom = PhysicalDomain.create((4, 50, 4), (True, False, True), scale_factors=(2 * math.pi, 1.0, 1.0e-3))
    lsc = LinearStabilityCalculation(Re=re, alpha=1.0, beta=0.0, n=50)
    u = lsc.calculate_transient_growth_initial_condition(dom, t, 60)
    u_hat = (u * (1e-5 / math.sqrt(u.energy()))).hat().get_data().cpu().numpy()
    st = O.make_stepper("perturbation", (4, 50, 4), 2 * math.pi, 1.0e-3, re, 0.01, linearise=True)
    u_t, _, _ = O.run(st, u_hat, int(t / 0.01))
    gain = st.g.energy(u_t) / st.g.energy(u_hat)
    assert abs(gain / lsc.calculate_transient_growth_max_energy(t, 60) - 1) < 1e-6
