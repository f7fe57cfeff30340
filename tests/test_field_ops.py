"""Field operators of the drop-in surface on the host: VectorField.curl/div
(field.py:917-948), FourierField.solve_poisson (field.py:3059-3083 with the
matrix of domain.py:857-889), PhysicalField.FromRandom (field.py:1281-1310)
and Equation.find_suitable_dt (equation.py:114-162)."""
import math

import numpy as np
import pytest
import torch

from jax_spectral_dns import _ops, seeds
from jax_spectral_dns.domain import PhysicalDomain
from jax_spectral_dns.equation import Equation
from jax_spectral_dns.field import FourierField, PhysicalField, VectorField

LX, LZ = 2 * np.pi, np.pi


def _dom(shape=(8, 33, 8)):
    return PhysicalDomain.create(shape, (True, False, True), scale_factors=(LX, 1.0, LZ), aliasing=3 / 2)


def test_div_of_seeded_velocity_vanishes():
    """The seeded fields are solenoidal: their divergence, in spectral and in
    physical space, is round-off."""
    shape = (8, 33, 8)
    dom = _dom(shape)
    u = VectorField.FromData(FourierField, dom, seeds.seeded_velocity_hat(shape, (LX, LZ), (3, 3), 1e-3, seed=4),
                             name="velocity_hat")
    scale = max(float(f.get_data().abs().max()) for f in u) * 4.0
    assert float(u.div().get_data().abs().max()) < 1e-10 * scale
    v = u.no_hat()
    d = v.div()
    assert d.energy() < 1e-20 * v.energy()
    assert d.name == "div_" + v.name


def test_curl_of_analytic_field():
    """u = (sin z (1 - y^2), 0, cos x (1 - y^2)): curl = (-2y cos x, cos z (1 - y^2) + sin x (1 - y^2), 2y sin z)."""
    dom = _dom((8, 33, 8))
    X = dom.mgrid
    fx = PhysicalField.FromFunc(dom, lambda X: np.sin(2 * X[2]) * (1 - X[1] ** 2))
    fy = PhysicalField.FromFunc(dom, lambda X: 0.0 * X[0])
    fz = PhysicalField.FromFunc(dom, lambda X: np.cos(X[0]) * (1 - X[1] ** 2))
    c = VectorField([fx, fy, fz], "u").curl()
    x, y, z = (np.asarray(m) for m in X)
    want = [-2 * y * np.cos(x), 2 * np.cos(2 * z) * (1 - y ** 2) + np.sin(x) * (1 - y ** 2), 2 * y * np.sin(2 * z)]
    for i in range(3):
        assert np.abs(c[i].get_data().cpu().numpy() - want[i]).max() < 1e-10
    # spectral fields give the same curl
    ch = VectorField([fx.hat(), fy.hat(), fz.hat()], "u_hat").curl()
    for i in range(3):
        assert np.abs(ch[i].no_hat().get_data().cpu().numpy() - want[i]).max() < 1e-10


def test_solve_poisson_matches_dense_matrix_and_analytic():
    """(D2 - k^2) p = f with p = 0 at the walls: the eigenbasis solve equals the
    reference's dense per-wavenumber inverse and an analytic solution."""
    shape = (8, 33, 8)
    dom = _dom(shape)
    t = _ops.operator_tables(dom.get_shape()[1])
    kx, kz = dom.hat().grid[0], dom.hat().grid[2]
    # analytic: p = sin(x) cos(2 z) (1 - y^2)^2 -> f = lap p
    P = lambda X: np.sin(X[0]) * np.cos(2 * X[2]) * (1 - X[1] ** 2) ** 2
    F = lambda X: np.sin(X[0]) * np.cos(2 * X[2]) * ((12 * X[1] ** 2 - 4) - 5 * (1 - X[1] ** 2) ** 2)
    f_hat = PhysicalField.FromFunc(dom, F).hat()
    p_hat = f_hat.solve_poisson()
    p_want = PhysicalField.FromFunc(dom, P).get_data().cpu().numpy()
    # interior rows solve the Poisson equation; the unit wall rows of the
    # reference's matrix carry the right-hand side's wall values through
    got = p_hat.no_hat().get_data().cpu().numpy()
    assert np.abs(got[:, 1:-1] - p_want[:, 1:-1]).max() < 1e-8
    assert torch.equal(p_hat.get_data()[:, [0, -1]], f_hat.get_data()[:, [0, -1]])
    # dense matrices as the reference assembles them
    ny = dom.get_shape()[1]
    eye_bc = np.eye(ny)
    eye_bc[0, 0] = eye_bc[-1, -1] = 0.0
    ymat = t.D @ t.D
    ymat[0, :] = 0.0
    ymat[:, 0] = 0.0
    ymat[0, 0] = 1.0
    ymat[-1, :] = 0.0
    ymat[:, -1] = 0.0
    ymat[-1, -1] = 1.0
    mat = np.array([[np.linalg.inv(-(a * a + b * b) * eye_bc + ymat) for b in kz] for a in kx])
    p_dense = f_hat.solve_poisson(mat)
    d = p_dense.get_data()
    assert float((p_hat.get_data() - d).abs().max()) < 1e-12 * float(d.abs().max())


def test_from_random_is_normalised_and_wall_free():
    dom = _dom((8, 33, 8))
    f = PhysicalField.FromRandom(dom, seed=3, energy_norm=2.5)
    assert abs(f.energy() / 2.5 - 1) < 1e-13
    data = f.get_data()
    assert float(data[:, 0, :].abs().max()) == 0.0 and float(data[:, -1, :].abs().max()) == 0.0
    g = PhysicalField.FromRandom(dom, seed=3, energy_norm=2.5)
    assert torch.equal(f.get_data(), g.get_data())


@pytest.mark.parametrize("end_time", [None, 15.0, 0.5, 1.0])
def test_find_suitable_dt(end_time):
    """The reference's rule, restated here in plain Python."""
    dom = _dom((8, 33, 8))
    U = (1.0, 0.3, 0.2)
    got = Equation.find_suitable_dt(dom, 0.5, U, end_time)
    dT = [abs(0.5 * (dom.get_extent(i) / dom.number_of_cells(i)) / U[i]) for i in range(3)]
    dt = 0.9 * min(dT)
    if end_time is not None:
        n = int(end_time / dt)

        def med(n):
            fs = []
            for i in range(1, int(n ** 0.5) + 1):
                if n % i == 0:
                    fs += [i, n // i]
            return sorted(fs)[len(fs) // 2]

        while math.sqrt(n) - n // med(n) > n // med(n):
            n += 1
        dt = end_time / n
    assert got == pytest.approx(dt, rel=1e-15)
