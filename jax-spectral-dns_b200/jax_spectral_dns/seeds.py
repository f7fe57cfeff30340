"""Seeded synthetic initial fields for the (v, omega_y) channel step.

Pure NumPy, host side. The construction follows the workload definition of the
benchmark configurations: for every admissible wavenumber pair (kx, kz) draw
complex Chebyshev coefficients c_n, d_n ~ N(0,1) + i N(0,1) damped by
exp(-n/8); evaluate on the Gauss-Lobatto points; multiply by (1-y^2)^2 for the
wall-normal velocity v and by (1-y^2) for the wall-normal vorticity omega_y so
that no-slip holds exactly; the series stop at n < Ny-4 (v) and n < Ny-2
(omega_y) so both products are polynomials of degree <= Ny-1, which the
collocation grid represents exactly (dv/dy then vanishes at the walls to
round-off and the field is divergence-free at every point); impose Hermitian symmetry F(-k) = conj F(k); then
recover (u, w) from continuity and the definition of omega_y exactly as the
reference does in ``NavierStokesVelVort.vort_yvel_to_vel``
(navier_stokes.py:1100-1123):

    u = (-i kx dv/dy + i kz omega) / (-(kx^2 + kz^2))
    w = (-i kz dv/dy - i kx omega) / (-(kx^2 + kz^2))

with the (0, 0) mode left at zero. Finally the field is scaled to the requested
kinetic energy E0 (``VectorField.energy`` semantics, field.py:607).

Arrays use the reference's spectral layout: (3, Mx, Ny, Mz) complex128, kx and
kz in FFT order [0..K, -K..-1], y index 0 at y = +1.
"""
from __future__ import annotations

import math

import numpy as np


def cheb_points(ny: int) -> np.ndarray:
    """Gauss-Lobatto points y_i = cos(pi / (Ny-1) * i), evaluated point by
    point in the same operation order as get_cheb_grid (domain.py:130-140)."""
    return np.array([np.cos(np.pi / (ny - 1) * i) for i in np.arange(ny)])


def cheb_diff_matrix(y: np.ndarray) -> np.ndarray:
    """First-order Chebyshev collocation matrix on the points y.

    Same construction as ``assemble_cheb_diff_mat`` (domain.py:155-163):
    off-diagonal entries c_i/c_j (-1)^(i+j) / (y_i - y_j), diagonal from the
    negative row sum.
    """
    n = len(y)
    c = np.ones(n)
    c[0] = c[-1] = 2.0
    c = c * (-1.0) ** np.arange(n)
    dy = y[:, None] - y[None, :]
    d = np.outer(c, 1.0 / c) / (dy + np.eye(n))
    # diagonal = -(sum of the off-diagonal row entries); accumulated column by
    # column in index order, the order the reference's builtin sum uses
    acc = np.zeros(n)
    for j in range(n):
        acc = acc + d[:, j]
    return d - np.diag(acc)


def fourier_wavenumbers(m: int, length: float) -> np.ndarray:
    """Wavenumbers in FFT order for M = 2K+1 modes on a period `length`
    (``FourierDomain.FromPhysicalDomain``, domain.py:791-848)."""
    k = m // 2
    idx = np.concatenate([np.arange(0, k + 1), np.arange(-k, 0)])
    return idx * (2.0 * np.pi / length)


def mode_counts(shape: tuple[int, int, int], aliasing: float = 1.5):
    """Fourier mode counts and reference physical grid sizes of
    ``Domain.create`` (domain.py:201-317) for a periodic-Chebyshev-periodic box.

    Returns ((Mx, Ny, Mz), (Px, Ny, Pz)).
    """
    modes = []
    phys = []
    for i, n in enumerate(shape):
        n = int(n)
        if i == 1:
            modes.append(n)
            phys.append(n)
            continue
        m = n if n % 2 != 0 else n + 1
        p = math.ceil(m * aliasing)
        p = p if p % 2 != 0 else p + 1
        # get_fourier_grid drops one point of an odd count
        p_grid = p - 1 if p % 2 != 0 else p
        modes.append(m)
        phys.append(p_grid)
    return tuple(modes), tuple(phys)


def spectral_energy(vel_hat: np.ndarray, phys_shape, lengths) -> float:
    """Kinetic energy of a spectral field with ``VectorField.energy`` semantics.

    E = 1/(2 V) * sum_x sum_z (Lx/Px)(Lz/Pz) sum_y w_y u^2 / 2 per component,
    evaluated by Parseval on the Hermitian part of the coefficients
    (field.py:1456-1475, domain.py:485-628). Exact for band-limited fields.
    """
    px, ny, pz = phys_shape
    lx, lz = lengths
    s = lx * lz / (4.0 * np.pi ** 2)
    w = cheb_integration_weights(ny)
    mx, mz = vel_hat.shape[1], vel_hat.shape[3]
    ix = (-np.arange(mx)) % mx
    iz = (-np.arange(mz)) % mz
    sym = 0.5 * (vel_hat + np.conj(vel_hat[:, ix][:, :, :, iz]))
    per_y = np.sum(np.abs(sym) ** 2, axis=(0, 1, 3))
    return float(0.25 * s * s / (px * pz) * np.dot(w, per_y))


def cheb_integration_weights(ny: int) -> np.ndarray:
    """Weights w with sum_y w_y f_y = int_{-1}^{1} f dy as the reference computes
    it: invert D with its first row/column replaced by the unit vector, apply it
    to f with the first entry zeroed, take (row 0) - (row Ny-1)
    (``Domain.integrate`` order 1 with bc_right, domain.py:485-628 and
    ``PhysicalField.definite_integral``, field.py:2618-2650)."""
    y = cheb_points(ny)
    d = cheb_diff_matrix(y)
    m = d.copy()
    m[0, :] = 0.0
    m[:, 0] = 0.0
    m[0, 0] = 1.0
    inv = np.linalg.inv(m)
    w = inv[0, :] - inv[-1, :]
    w[0] = 0.0
    return w


def seeded_velocity_hat(
    shape: tuple[int, int, int],
    lengths: tuple[float, float],
    kmax: tuple[int, int],
    e0: float,
    seed: int,
    aliasing: float = 1.5,
) -> np.ndarray:
    """Solenoidal, no-slip random perturbation in the reference's spectral layout.

    shape   -- (Nx, Ny, Nz) as passed to ``PhysicalDomain.create``
    lengths -- (Lx, Lz)
    kmax    -- largest |mode index| populated in x and z
    e0      -- target kinetic energy
    """
    (mx, ny, mz), phys = mode_counts(shape, aliasing)
    lx, lz = lengths
    rng = np.random.Generator(np.random.PCG64(seed))
    y = cheb_points(ny)
    d = cheb_diff_matrix(y)
    n = np.arange(ny)
    tmat = np.cos(np.outer(np.arccos(np.clip(y, -1.0, 1.0)), n))  # T_n(y_i)
    damp = np.exp(-n / 8.0)
    kxs = fourier_wavenumbers(mx, lx)
    kzs = fourier_wavenumbers(mz, lz)
    kx_max_idx = mx // 2
    kz_max_idx = mz // 2
    v = np.zeros((mx, ny, mz), dtype=np.complex128)
    om = np.zeros((mx, ny, mz), dtype=np.complex128)

    def idx(i: int, m: int) -> int:
        return i % m

    for ix in range(-min(kmax[0], kx_max_idx), min(kmax[0], kx_max_idx) + 1):
        for iz in range(-min(kmax[1], kz_max_idx), min(kmax[1], kz_max_idx) + 1):
            if ix == 0 and iz == 0:
                continue
            # one draw per Hermitian pair: the "positive" representative
            if ix < 0 or (ix == 0 and iz < 0):
                continue
            c = (rng.standard_normal(ny) + 1j * rng.standard_normal(ny)) * damp
            dd = (rng.standard_normal(ny) + 1j * rng.standard_normal(ny)) * damp
            c[ny - 4:] = 0.0
            dd[ny - 2:] = 0.0
            vy = (1.0 - y ** 2) ** 2 * (tmat @ c)
            oy = (1.0 - y ** 2) * (tmat @ dd)
            a, b = idx(ix, mx), idx(iz, mz)
            v[a, :, b] = vy
            om[a, :, b] = oy
            a2, b2 = idx(-ix, mx), idx(-iz, mz)
            v[a2, :, b2] = np.conj(vy)
            om[a2, :, b2] = np.conj(oy)
    vel = np.zeros((3, mx, ny, mz), dtype=np.complex128)
    vel[1] = v
    for a in range(mx):
        for b in range(mz):
            kx, kz = kxs[a], kzs[b]
            k2 = kx * kx + kz * kz
            if k2 == 0.0:
                continue
            dv = d @ v[a, :, b]
            vel[0, a, :, b] = (-1j * kx * dv + 1j * kz * om[a, :, b]) / (-k2)
            vel[2, a, :, b] = (-1j * kz * dv - 1j * kx * om[a, :, b]) / (-k2)
    vel[:, :, 0, :] = 0.0
    vel[:, :, -1, :] = 0.0
    e = spectral_energy(vel, phys, lengths)
    if e > 0.0:
        vel *= math.sqrt(e0 / e)
    return vel


def reichardt_profile(y: np.ndarray, re_tau: float) -> np.ndarray:
    """Reichardt's law of the wall mirrored about y = 0:
    u+(y+) = 2.5 ln(1 + 0.4 y+) + 7.8 (1 - exp(-y+/11) - (y+/11) exp(-y+/3)),
    y+ = (1 - |y|) Re_tau."""
    yp = (1.0 - np.abs(y)) * re_tau
    return 2.5 * np.log1p(0.4 * yp) + 7.8 * (1.0 - np.exp(-yp / 11.0) - (yp / 11.0) * np.exp(-yp / 3.0))


def turbulent_channel_hat(
    shape: tuple[int, int, int],
    lengths: tuple[float, float],
    re_tau: float,
    kmax: tuple[int, int],
    seed: int,
    aliasing: float = 1.5,
    peak_fraction: float = 0.1,
) -> np.ndarray:
    """Reichardt mean profile in the (0,0) streamwise mode plus a seeded
    solenoidal perturbation whose largest velocity component value on the
    reference physical grid is `peak_fraction` of the centreline velocity."""
    (mx, ny, mz), (px, _, pz) = mode_counts(shape, aliasing)
    lx, lz = lengths
    y = cheb_points(ny)
    u_mean = reichardt_profile(y, re_tau)
    u_cl = float(u_mean.max())
    vel = seeded_velocity_hat(shape, lengths, kmax, 1.0, seed, aliasing)
    s = lx * lz / (4.0 * np.pi ** 2)
    peak = max(float(np.abs(_physical(vel[c], px, pz, s)).max()) for c in range(3))
    if peak > 0.0:
        vel *= peak_fraction * u_cl / peak
    # a constant-in-(x,z) physical field c maps to c * sqrt(Px Pz) / s at (0,0)
    vel[0, 0, :, 0] += u_mean * math.sqrt(px * pz) / s
    return vel


def _physical(f_hat: np.ndarray, px: int, pz: int, s: float) -> np.ndarray:
    """Physical values of one spectral field on the reference grid (zero
    padding, ortho inverse FFT, real part, times s: domain.py:1167-1242)."""
    mx, ny, mz = f_hat.shape
    kx, kz = mx // 2, mz // 2
    full = np.zeros((px, ny, pz), dtype=np.complex128)
    ix = np.concatenate([np.arange(kx + 1), np.arange(px - kx, px)])
    iz = np.concatenate([np.arange(kz + 1), np.arange(pz - kz, pz)])
    full[np.ix_(ix, np.arange(ny), iz)] = f_hat
    return np.fft.ifftn(full, axes=(0, 2), norm="ortho").real * s


def laminar_base_hat(shape, lengths, u_max: float = 1.0, aliasing: float = 1.5) -> np.ndarray:
    """Spectral coefficients of the laminar base flow U = u_max (1 - y^2)
    (navier_stokes_perturbation.py:351-380) in the reference normalisation."""
    (mx, ny, mz), (px, _, pz) = mode_counts(shape, aliasing)
    lx, lz = lengths
    s = lx * lz / (4.0 * np.pi ** 2)
    y = cheb_points(ny)
    out = np.zeros((3, mx, ny, mz), dtype=np.complex128)
    out[0, 0, :, 0] = u_max * (1.0 - y ** 2) * math.sqrt(px * pz) / s
    return out
