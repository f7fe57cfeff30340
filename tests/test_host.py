"""Host-side logic: seeds, operator tables, domain shapes, field transforms."""
import math

import numpy as np
import pytest
import torch

import jsd_oracle as O
from jax_spectral_dns import _ops, seeds
from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.field import FourierField, PhysicalField, VectorField
from conftest import golden, rel


@pytest.mark.parametrize("shape", [(8, 65, 4), (32, 65, 32), (48, 65, 48), (128, 129, 128), (4, 24, 12)])
def test_domain_shapes_match_reference_rules(shape):
    modes, phys = seeds.mode_counts(shape)
    g = O.Grid(shape, 2 * np.pi, np.pi)
    assert modes == g.modes and phys == g.phys
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(2 * np.pi, 1.0, np.pi))
    assert dom.get_shape() == modes and dom.get_shape_aliasing() == phys
    assert np.array_equal(dom.hat().grid[0], g.kx) and np.array_equal(dom.hat().grid[2], g.kz)
    assert np.array_equal(dom.diff_mats[1], g.D)


def test_mode_count_3_mod_4_rejected():
    with pytest.raises(NotImplementedError, match="3 mod 4"):
        PhysicalDomain.create((6, 24, 8), (True, False, True))


def test_seed_is_hermitian_solenoidal_noslip():
    shape, lx, lz = (16, 33, 16), 2 * np.pi, np.pi
    u = seeds.seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-3, seed=7)
    g = O.Grid(shape, lx, lz)
    ix = (-np.arange(g.mx)) % g.mx
    iz = (-np.arange(g.mz)) % g.mz
    assert np.abs(u - np.conj(u[:, ix][:, :, :, iz])).max() < 1e-15 * np.abs(u).max()
    div = g.divergence(u)
    assert np.abs(div).max() < 1e-10 * np.abs(u).max() * g.kx.max()
    assert np.abs(u[:, :, [0, -1], :]).max() == 0.0
    assert abs(g.energy(u) / 1e-3 - 1) < 1e-12


def test_spectral_energy_matches_physical_quadrature():
    d = golden("ns_cmf_9x33x9")
    g = O.Grid(tuple(d["shape"]), *d["lengths"])
    e = seeds.spectral_energy(d["u1"], g.phys, tuple(d["lengths"]))
    assert abs(e / g.energy(d["u1"]) - 1) < 1e-13


@pytest.mark.parametrize("ny", [24, 33, 65, 129])
def test_eigenbasis_tables(ny):
    t = _ops.operator_tables(ny)
    A = t.D2[1:-1, 1:-1]
    assert np.abs(t.V @ np.diag(t.lam) @ t.Vinv - A).max() < 1e-9 * np.abs(A).max()
    assert np.all(t.lam < 0)
    J = t.V[::-1, :]
    assert np.abs(J - t.V * t.sgn).max() < 1e-8
    assert np.allclose(t.w0, t.D[0, 1:-1] @ t.V) and np.allclose(t.c0, t.Vinv @ t.D2[1:-1, 0])
    # integration weights integrate polynomials exactly
    y = seeds.cheb_points(ny)
    assert abs(t.y_weights @ (y ** 2) - 2 / 3) < 1e-12


@pytest.mark.parametrize("ny,k2", [(33, 0.0), (33, 5.0), (65, 1.0), (129, 64.0)])
def test_eigenbasis_solves_match_dense_inverses(ny, k2):
    """Diagonal solves in the D2_int eigenbasis reproduce the reference's dense
    Helmholtz and Poisson inverses (navier_stokes.py:920-1022, domain.py:857-889)."""
    t = _ops.operator_tables(ny)
    re, dt = 180.0, 0.002
    n = ny - 2
    L = t.D2[1:-1, 1:-1] - k2 * np.eye(n)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(n)
    for beta in O.RK_BETA:
        ref = np.linalg.solve(np.eye(n) - beta * dt / re * L, x)
        mine = t.V @ ((t.Vinv @ x) / (1 - beta * dt / re * (t.lam - k2)))
        assert rel(mine, ref) < 1e-13
    ref = np.linalg.solve(L, x)
    mine = t.V @ ((t.Vinv @ x) / (t.lam - k2))
    assert rel(mine, ref) < 1e-11


def test_mean_flow_matrices_match_oracle():
    g = O.Grid((8, 33, 8), 4 * np.pi, 4 * np.pi / 3)
    st = O.Stepper(g, 180.0, 0.002, kind="ns")
    rhs, lhs = _ops.mean_flow_matrices(33, 180.0, 0.002)
    for s in range(3):
        assert np.array_equal(rhs[s], st.rhs_ns[s])
        assert np.abs(lhs[s] - st.lhs_inv_ns[s]).max() < 1e-14


@pytest.mark.parametrize("m,n", [(5, 7), (9, 14), (33, 49), (49, 75), (65, 98), (129, 196)])
def test_fft_size_choice(m, n):
    assert _ops.smooth_fft_size(m) == n
    assert n >= 3 * (m // 2) + 1


def test_field_transforms_match_oracle():
    d = golden("nonlin_pert_9x33x9")
    shape, (lx, lz) = tuple(d["shape"]), d["lengths"]
    g = O.Grid(shape, lx, lz)
    dom = PhysicalDomain.create(shape, (True, False, True), scale_factors=(lx, 1.0, lz))
    f = FourierField(dom, torch.as_tensor(d["u1"][0]))
    phys = f.no_hat()
    assert rel(phys.data.cpu().numpy(), g.no_hat(d["u1"][0])) < 1e-14
    back = phys.hat()
    assert rel(back.data.cpu().numpy(), g.hat(g.no_hat(d["u1"][0]))) < 1e-14
    vf = VectorField.FromData(FourierField, dom, torch.as_tensor(d["u1"]))
    assert abs(vf.no_hat().energy() / g.energy(d["u1"]) - 1) < 1e-13


def test_reichardt_channel_seed():
    shape, lx, lz = (16, 33, 16), 4 * np.pi, 4 * np.pi / 3
    u = seeds.turbulent_channel_hat(shape, (lx, lz), 180.0, (4, 4), seed=1)
    g = O.Grid(shape, lx, lz)
    mean = g.no_hat(u[0]).mean(axis=(0, 2))
    prof = seeds.reichardt_profile(g.y, 180.0)
    assert np.abs(mean - prof).max() < 1e-10 * prof.max()


def test_vort_yvel_to_vel_matches_reference():
    """NavierStokesVelVort.vort_yvel_to_vel / smooth_and_enforce_bc_vel_y against
    the reference's own outputs (tests/golden/vort_yvel_9x33x9.npz)."""
    from jax_spectral_dns.navier_stokes import NavierStokesVelVort as NS

    d = golden("vort_yvel_9x33x9")
    dom = PhysicalDomain.create(tuple(int(x) for x in d["shape"]), (True, False, True),
                                scale_factors=(d["lengths"][0], 1.0, d["lengths"][1]))
    out3 = NS.vort_yvel_to_vel(dom, d["vort"], d["vel_y"], d["ux00"], d["uz00"]).cpu().numpy()
    assert np.linalg.norm(out3 - d["out3"]) < 1e-12 * np.linalg.norm(d["out3"])
    out2 = NS.vort_yvel_to_vel(dom, None, d["vel_y"], d["ux00"], None, two_d=True).cpu().numpy()
    assert np.linalg.norm(out2 - d["out2"]) < 1e-12 * np.linalg.norm(d["out2"])
    sm = NS.smooth_and_enforce_bc_vel_y(dom, d["slice_in"]).cpu().numpy()
    assert np.linalg.norm(sm - d["slice_out"]) < 1e-12 * np.linalg.norm(d["slice_out"])
    sm10 = NS.smooth_and_enforce_bc_vel_y(dom, d["slice_in"], M=10).cpu().numpy()
    assert np.linalg.norm(sm10 - d["slice_out_m10"]) < 1e-12 * np.linalg.norm(d["slice_out_m10"])
    # the smoothed profiles satisfy v = dv/dy = 0 at both walls
    from jax_spectral_dns.domain import assemble_cheb_diff_mat, get_cheb_grid
    dm = assemble_cheb_diff_mat(get_cheb_grid(33))
    v = out3[1]
    assert np.abs(v[:, [0, -1], :]).max() < 1e-12 * np.abs(v).max()
    assert np.abs(np.einsum("lj,ijk->ilk", dm, v)[:, [0, -1], :]).max() < 1e-9 * np.abs(v).max()
