"""Host-side FP64 operator tables for one channel box (built once per plan).

The reference assembles dense per-wavenumber inverses for every RK stage
(``prepare_assemble_rk_matrices``, navier_stokes.py:920-1022, and
``assemble_poisson_matrix``, domain.py:857-889): (3, Mx, Mz, Ny, Ny) complex
arrays. All of those operators are real and are rational functions of the
interior second-derivative matrix D2_int = D2[1:-1, 1:-1] and of k^2, so with
the eigen-decomposition D2_int = V diag(lam) V^-1 they become diagonal:

  Helmholtz  (I - beta dt/Re (D2 - k^2))^-1   ->  1 / (1 - beta dt/Re (lam - k^2))
  explicit   (I + alpha dt/Re (D2 - k^2))     ->  1 + alpha dt/Re (lam - k^2)
  Poisson    (D2 - k^2)^-1                    ->  1 / (lam - k^2)

D2_int commutes with the reflection y -> -y, so each eigenvector is even or
odd (``sgn``); the influence solution v_b = flip(v_a) is then sgn * v_a in
eigen-coordinates. The (0,0) mean-flow system keeps the reference's own
2Ny x 2Ny matrices.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .seeds import cheb_diff_matrix, cheb_points

RK_ALPHA = (29 / 96, -3 / 40, 1 / 6)
RK_BETA = (37 / 160, 5 / 24, 1 / 6)


def _bc_hom(mat: np.ndarray) -> np.ndarray:
    """First/last rows and columns -> unit (enforce_homogeneous_dirichlet, domain.py:375-397)."""
    out = mat.copy()
    out[0, :] = 0.0
    out[:, 0] = 0.0
    out[0, 0] = 1.0
    out[-1, :] = 0.0
    out[:, -1] = 0.0
    out[-1, -1] = 1.0
    return out


@dataclass
class OperatorTables:
    ny: int
    D: np.ndarray
    D2: np.ndarray
    V: np.ndarray
    Vinv: np.ndarray
    lam: np.ndarray
    sgn: np.ndarray
    c0: np.ndarray
    cN: np.ndarray
    w0: np.ndarray
    wN: np.ndarray
    y_weights: np.ndarray


_cache: dict = {}


def operator_tables(ny: int) -> OperatorTables:
    if ny in _cache:
        return _cache[ny]
    y = cheb_points(ny)
    D = cheb_diff_matrix(y)
    D2 = D @ D
    A = D2[1:-1, 1:-1]
    lam, V = np.linalg.eig(A)
    if np.abs(np.imag(lam)).max() > 0 or np.abs(np.imag(V)).max() > 0:
        raise RuntimeError("interior D2 has a complex spectrum; eigenbasis solve not applicable")
    lam = np.real(lam)
    V = np.real(V)
    order = np.argsort(lam)
    lam, V = lam[order], V[:, order]
    V = V / np.linalg.norm(V, axis=0)
    Vinv = np.linalg.inv(V)
    # parity of each eigenvector under the reflection y -> -y
    sgn = np.sign(np.sum(V[::-1, :] * V, axis=0))
    if np.abs(V[::-1, :] - V * sgn).max() > 1e-8:
        raise RuntimeError("eigenvectors of D2_int are not of definite parity")
    c0 = Vinv @ D2[1:-1, 0]
    cN = Vinv @ D2[1:-1, -1]
    w0 = D[0, 1:-1] @ V
    wN = D[-1, 1:-1] @ V
    # integration weights: inv(D with first row/col unit), row 0 - row N-1
    m = D.copy()
    m[0, :] = 0.0
    m[:, 0] = 0.0
    m[0, 0] = 1.0
    inv = np.linalg.inv(m)
    yw = inv[0, :] - inv[-1, :]
    yw[0] = 0.0
    t = OperatorTables(ny, D, D2, V, Vinv, lam, sgn, c0, cN, w0, wN, yw)
    _cache[ny] = t
    return t


def mean_flow_matrices(ny: int, re_tau: float, dt: float):
    """(0,0) explicit matrices and implicit inverses for the 3 RK stages, built
    as prepare_assemble_rk_matrices does (navier_stokes.py:1000-1022): block
    diagonal diag(D2_hom, D2_hom)/Re with the homogeneous-Dirichlet rows and
    columns enforced on the 2Ny system as a whole."""
    t = operator_tables(ny)
    D2_hom = _bc_hom(t.D2)
    Z = np.zeros((ny, ny))
    L_ns = 1 / re_tau * np.block([[D2_hom, Z], [Z, D2_hom]])
    I_ns = np.eye(2 * ny)
    rhs, lhs_inv = [], []
    for st in range(3):
        rhs.append(_bc_hom(I_ns + RK_ALPHA[st] * dt * L_ns))
        lhs_inv.append(np.linalg.inv(_bc_hom(I_ns - RK_BETA[st] * dt * L_ns)))
    return np.ascontiguousarray(np.array(rhs)), np.ascontiguousarray(np.array(lhs_inv))


# sides S of the square FFT lengths S * S that have register-resident kernels
SQUARE_FFT_SIDES = (3, 4, 5, 7, 10, 14)


def device_fft_size(m: int) -> int:
    """FFT length the device uses for m modes: the smallest S * S >= 3K + 1 with
    a register-resident square-FFT kernel, else the smallest 2,3,5,7-smooth
    length >= 3K + 1."""
    need = 3 * (m // 2) + 1
    for s in SQUARE_FFT_SIDES:
        if s * s >= need:
            return s * s
    return smooth_fft_size(m)


def smooth_fft_size(m: int) -> int:
    """Smallest length >= 3K + 1 (K = m // 2) whose prime factors are 2, 3, 5, 7;
    any such length dealiases quadratic products exactly."""
    n = 3 * (m // 2) + 1
    while True:
        r = n
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return n
        n += 1


def fourier_scale(lx: float, lz: float) -> float:
    return (lx / (2 * math.pi)) * (lz / (2 * math.pi))
