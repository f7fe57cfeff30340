"""Linear stability and optimal transient growth of plane channel flow.

Drop-in for ``LinearStabilityCalculation`` of dakling/jax-spectral-dns
(linear_stability_calculation.py:34-638). For one wavenumber pair (alpha,
beta) it discretises the linearised Navier-Stokes equations about U(y)
(default Poiseuille 1 - y^2) in wall-conforming Chebyshev bases, solves the
generalised eigenproblem A q = lambda B q, and from the leading eigenmodes
builds the energy-norm propagator F exp(Lambda T) F^-1 whose largest
singular value squared is the optimal energy gain at time T and whose right
singular vector gives the optimal initial condition. That initial condition
seeds the transient-growth checks of the channel step (the reference's
``run_transient_growth``, examples.py:1274-1413).

What is the same as the reference, and why:
* the bases (cheb.py:12-49): u, w in phi_a(k) = T_{2k+3} - T_{2k+1}, v in
  phi_s(k) = T_{2k+2} - T_{2k}, p in T_{2k+1}, collocated at the first half
  of the Gauss-Lobatto points (symmetric form, the reference's only active
  one: ``self.symm = True``), or phi(k) = T_{k+2} - T_k and T_k on all points;
  the 4 x 4 block layout of A and B (linear_stability_calculation.py:98-185);
  evaluated with NumPy's Chebyshev series as in the reference, so A and B
  agree with it to the last bit up to signed zeros;
* the eigen-solve (scipy.linalg.eig on (A, B)), the filter Re(lambda) <= 1 and
  the descending sort by Re(lambda) (:188-214), since the mode order defines
  which modes enter the propagator;
* the energy Gram matrix C, its Cholesky factor F, the SVD of F Sigma F^-1
  and coeffs = F^-1 v_1 (:437-536).
What differs:
* the Gram integrals of basis pairs are exact (Chebyshev product identity
  int T_m T_n = (I_{m+n} + I_{|m-n|}) / 2, I_k = 2 / (1 - k^2) for even k)
  where the reference calls adaptive quadrature per pair (scipy quad);
* C is one matrix product per velocity block instead of a five-fold loop;
* gains for many horizons (``transient_growth_gains`` and the ``Ts`` option)
  are one batched SVD on the field device (the GPU when present) instead of
  one SVD per horizon;
* nothing is read from or written to files: the reference caches fields and
  eigenpairs in ./fields (HDF5 / pickle); here every call computes, and the
  ``save`` flags keep results in memory only.
"""
from __future__ import annotations

import warnings
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
from numpy.polynomial import chebyshev as npcheb
from scipy.linalg import cholesky, eig

from .domain import PhysicalDomain, _default_device, assemble_cheb_diff_mat, get_cheb_grid
from .field import PhysicalField, VectorField

# Chebyshev orders (high, low) of the basis function number k, per basis kind:
# the function is T_high - T_low (low < 0: T_high alone).
_BASIS_ORDERS = {
    "a": lambda k: (2 * k + 3, 2 * k + 1),  # antisymmetric, vanishes at y = +-1
    "s": lambda k: (2 * k + 2, 2 * k),      # symmetric, vanishes at y = +-1
    "p": lambda k: (2 * k + 1, -1),          # pressure, odd
    "full": lambda k: (k + 2, k),            # general, vanishes at y = +-1
    "cheb": lambda k: (k, -1),               # plain T_k
}


def _unit_series(order: int) -> npcheb.Chebyshev:
    coef = np.zeros(order + 1)
    coef[order] = 1.0
    return npcheb.Chebyshev(coef)


def basis_function(kind: str, k: int, deriv: int = 0) -> npcheb.Chebyshev:
    """Basis function number k of the given kind, differentiated ``deriv``
    times, as a NumPy Chebyshev series (cheb.py:12-49: ``phi_a``, ``phi_s``,
    ``phi_pressure``, ``phi``, ``cheby``)."""
    hi, lo = _BASIS_ORDERS[kind](k)
    series = _unit_series(hi).deriv(deriv)
    if lo >= 0:
        series = series - _unit_series(lo).deriv(deriv)
    return series


def basis_matrix(kind: str, n: int, ys: np.ndarray, deriv: int = 0) -> np.ndarray:
    """(len(ys), n) values of basis functions 0..n-1 at the points ys."""
    ys = np.asarray(ys, dtype=np.float64)
    out = np.empty((len(ys), n))
    for k in range(n):
        out[:, k] = basis_function(kind, k, deriv)(ys)
    return out


def _cheb_integrals(max_order: int) -> np.ndarray:
    """J[m, n] = int_{-1}^{1} T_m T_n dy for m, n <= max_order."""
    k = np.arange(2 * max_order + 1)
    ik = np.zeros(len(k))
    ik[::2] = 2.0 / (1.0 - k[::2].astype(np.float64) ** 2)
    m = np.arange(max_order + 1)
    return 0.5 * (ik[m[:, None] + m[None, :]] + ik[np.abs(m[:, None] - m[None, :])])


def gram_matrix(kind: str, n: int) -> np.ndarray:
    """G[p, q] = int_{-1}^{1} f_p f_q dy for basis functions 0..n-1 of a kind.
    For the symmetric kinds the integrand is even, so this equals the
    reference's 2 int_0^1 (linear_stability_calculation.py:446-455)."""
    orders = [_BASIS_ORDERS[kind](k) for k in range(n)]
    top = max(hi for hi, _ in orders)
    coef = np.zeros((n, top + 1))
    for k, (hi, lo) in enumerate(orders):
        coef[k, hi] += 1.0
        if lo >= 0:
            coef[k, lo] -= 1.0
    g = coef @ _cheb_integrals(top) @ coef.T
    return 0.5 * (g + g.T)


class LinearStabilityCalculation:
    """Orr-Sommerfeld-Squire analysis of one wavenumber pair (alpha, beta) at
    Reynolds number Re with n Chebyshev collocation points
    (linear_stability_calculation.py:34-96)."""

    def __init__(self, Re: float = 180.0, alpha: float = 3.25, beta: float = 0.0, n: int = 50,
                 U_max: Optional[float] = None, U_base: Optional[np.ndarray] = None):
        self.Re = Re
        self.alpha = alpha
        self.beta = beta
        self.n = n
        self.A: Optional[np.ndarray] = None
        self.B: Optional[np.ndarray] = None
        self.eigenvalues: Optional[np.ndarray] = None
        self.eigenvectors: Optional[List[np.ndarray]] = None
        self.C: Optional[np.ndarray] = None
        self.ys = get_cheb_grid(n)
        self.diff_mat = assemble_cheb_diff_mat(self.ys)
        self.velocity_field_: Optional[VectorField] = None
        self.S: Optional[np.ndarray] = None
        self.coeffs: Optional[np.ndarray] = None
        self.Gs: Optional[np.ndarray] = None
        self.symm = True
        if U_base is not None:
            self.U_base = np.asarray(U_base, dtype=np.float64)
        elif U_max is not None:
            self.U_base = U_max * (1.0 - self.ys ** 2)
        else:
            self.U_base = 1.0 - self.ys ** 2

    # ------------------------------------------------------------------ eigen
    def _kinds(self) -> Tuple[str, str, str]:
        """Basis kinds of (u and w, v, p)."""
        return ("a", "s", "p") if self.symm else ("full", "full", "cheb")

    def number_of_basis_functions(self) -> int:
        return self.n // 2 if self.symm else self.n

    def assemble_matrix_fast(self) -> Tuple[np.ndarray, np.ndarray]:
        """A and B of A q = lambda B q, q = (u, v, w, p) basis coefficients;
        rows: x, y, z momentum and continuity at the collocation points
        (linear_stability_calculation.py:98-185)."""
        ys = self.ys[: self.n // 2] if self.symm else self.ys
        n = len(ys)
        ku, kv, kp = self._kinds()
        u, d2u = basis_matrix(ku, n, ys, 0), basis_matrix(ku, n, ys, 2)
        v, dv, d2v = basis_matrix(kv, n, ys, 0), basis_matrix(kv, n, ys, 1), basis_matrix(kv, n, ys, 2)
        p, dp = basis_matrix(kp, n, ys, 0), basis_matrix(kp, n, ys, 1)
        w, d2w = u, d2u
        U = self.U_base[:n, None]
        dU = (self.diff_mat @ self.U_base)[:n, None]
        alpha, beta, re = self.alpha, self.beta, self.Re
        ksq = alpha ** 2 + beta ** 2
        mi = -1j
        A = np.zeros((4 * n, 4 * n), dtype=complex)
        B = np.zeros((4 * n, 4 * n), dtype=complex)

        def blk(mat, eq, var, value):
            mat[eq * n:(eq + 1) * n, var * n:(var + 1) * n] = value

        blk(B, 0, 0, u)
        blk(A, 0, 0, mi * alpha * U * u + 1 / re * (d2u - ksq * u))
        blk(A, 0, 1, v * -dU)
        blk(A, 0, 3, mi * alpha * p)
        blk(B, 1, 1, v)
        blk(A, 1, 1, mi * alpha * U * v + 1 / re * (d2v - ksq * v))
        blk(A, 1, 3, -dp)
        blk(B, 2, 2, w)
        blk(A, 2, 2, mi * alpha * U * w + 1 / re * (d2w - ksq * w))
        blk(A, 2, 3, mi * beta * p)
        blk(A, 3, 0, 1j * alpha * u)
        blk(A, 3, 1, dv)
        blk(A, 3, 2, 1j * beta * w)
        self.A, self.B = A, B
        return A, B

    def calculate_eigenvalues(self, save: bool = False) -> Tuple[np.ndarray, List[np.ndarray]]:
        """Finite eigenpairs with Re(lambda) <= 1, sorted by Re(lambda)
        descending (linear_stability_calculation.py:188-214)."""
        if self.A is None or self.B is None:
            self.assemble_matrix_fast()
        vals, vecs = eig(self.A, self.B)
        keep = [j for j in range(len(vals)) if vals[j].real <= 1]
        order = sorted(keep, key=lambda j: vals[j].real, reverse=True)
        self.eigenvalues = np.array([vals[j] for j in order])
        self.eigenvectors = [vecs[:, j] for j in order]
        if save:
            _no_files("eigenpairs")
        return self.eigenvalues, self.eigenvectors

    # -------------------------------------------------------------- fields
    def _y_profiles(self, domain: PhysicalDomain, evec: np.ndarray):
        """u, v, w of a coefficient vector on the domain's y points
        (linear_stability_calculation.py:268-309)."""
        u_c, v_c, w_c, _ = np.split(np.asarray(evec), 4)
        n = u_c.shape[0]
        ys = np.asarray(domain.grid[1])
        ku, kv, _ = self._kinds()
        pu = basis_matrix(ku, n, ys)
        pv = pu if kv == ku else basis_matrix(kv, n, ys)
        return pu @ u_c, pv @ v_c, pu @ w_c

    def y_slice_to_3d_field(self, domain: PhysicalDomain, y_slice_i, factor=1.0) -> np.ndarray:
        """Re(factor exp(i alpha x) f(y) exp(i beta z)) on the domain grid
        (linear_stability_calculation.py:311-332)."""
        ex = np.exp(1j * (self.alpha * np.asarray(domain.grid[0])))
        ez = np.exp(1j * (self.beta * np.asarray(domain.grid[2])))
        return (factor * (np.asarray(y_slice_i)[None, :, None] * ex[:, None, None] * ez[None, None, :])).real

    def velocity_field_from_y_slice(self, domain: PhysicalDomain, y_slice, factor=1.0) -> VectorField:
        names = ("velocity_pert_x", "velocity_pert_y", "velocity_pert_z")
        fields = [PhysicalField(domain, self.y_slice_to_3d_field(domain, y_slice[i], factor), name=names[i])
                  for i in range(3)]
        self.velocity_field_ = VectorField(fields)
        return self.velocity_field_

    def velocity_field(self, domain: PhysicalDomain, evec: np.ndarray, factor=1.0) -> VectorField:
        return self.velocity_field_from_y_slice(domain, self._y_profiles(domain, evec), factor=factor)

    def velocity_field_single_mode(self, domain: PhysicalDomain, mode: int = 0, factor=1.0,
                                   recompute_partial: bool = False, recompute_full: bool = False,
                                   save: bool = False) -> VectorField:
        """Velocity of eigenmode ``mode`` (linear_stability_calculation.py:224-266)."""
        if recompute_full or self.eigenvectors is None:
            self.calculate_eigenvalues()
        if save:
            _no_files("mode fields")
        return self.velocity_field(domain, self.eigenvectors[mode], factor)

    def energy_over_time(self, domain: PhysicalDomain, mode: int = 0, eps: float = 1.0
                         ) -> Tuple[Callable[[float, Optional[int]], float], complex]:
        """E(t) of eigenmode ``mode`` scaled by eps, growing like
        exp(2 Re(lambda) t) (linear_stability_calculation.py:373-429)."""
        if self.eigenvalues is None:
            self.calculate_eigenvalues()
        if self.velocity_field_ is None:
            self.velocity_field(domain, self.eigenvectors[mode])
        lam = self.eigenvalues[mode]
        vel = self.velocity_field_

        def out(t: float, dim: Optional[int] = None) -> float:
            g = float(np.exp(lam.real * t))
            dims = range(3) if dim is None else [dim]
            return eps ** 2 * sum((vel[d] * g).energy() for d in dims)

        return out, lam

    # ------------------------------------------------------ transient growth
    def energy_gram(self, number_of_modes: int) -> np.ndarray:
        """C[j, k] = energy inner product of eigenmodes j and k (Hermitian,
        real diagonal) (linear_stability_calculation.py:437-485)."""
        if self.eigenvalues is None or self.eigenvectors is None:
            self.calculate_eigenvalues()
        m = min(number_of_modes, len(self.eigenvectors))
        n = self.number_of_basis_functions()
        ev = np.array(self.eigenvectors[:m]).T  # (4n, m)
        ku, kv, _ = self._kinds()
        ga, gs = gram_matrix(ku, n), gram_matrix(kv, n)
        c = np.zeros((m, m), dtype=complex)
        for blk, g in enumerate((ga, gs, ga)):
            e = ev[blk * n:(blk + 1) * n]
            c += e.conj().T @ g @ e
        c = np.triu(c) + np.triu(c, 1).conj().T
        c[np.diag_indices(m)] = c.diagonal().real
        self.C = c
        return c

    def _propagator_factors(self, number_of_modes: int):
        c = self.energy_gram(number_of_modes)
        m = c.shape[0]
        f = cholesky(c, lower=False)
        return self.eigenvalues[:m], f, np.linalg.inv(f)

    def transient_growth_gains(self, Ts: Sequence[float], number_of_modes: int,
                               device: Optional[torch.device] = None) -> np.ndarray:
        """Optimal energy gain G(t) = ||F exp(Lambda t) F^-1||_2^2 for every t
        in Ts, as one batched SVD on ``device`` (default: the field device)."""
        evs, f, f_inv = self._propagator_factors(number_of_modes)
        dev = device or _default_device()
        ts = torch.as_tensor(np.asarray(Ts, dtype=np.float64), device=dev)
        lam = torch.as_tensor(evs, dtype=torch.complex128, device=dev)
        ft = torch.as_tensor(f, dtype=torch.complex128, device=dev)
        fi = torch.as_tensor(f_inv, dtype=torch.complex128, device=dev)
        sig = torch.exp(lam[None, :] * ts[:, None].to(torch.complex128))  # (T, m)
        mats = ft[None] * sig[:, None, :] @ fi[None]
        s = torch.linalg.svdvals(mats)
        return (s[:, 0] ** 2).cpu().numpy()

    def calculate_transient_growth_svd(self, T: float, number_of_modes: int, save: bool = False,
                                       recompute: bool = False, Ts: Optional[List[float]] = None
                                       ) -> Tuple[np.ndarray, np.ndarray]:
        """Singular values of F exp(Lambda T) F^-1 and the coefficients
        F^-1 v_1 of the optimal initial condition in the eigenmode basis
        (linear_stability_calculation.py:431-536)."""
        if recompute or self.eigenvalues is None or self.eigenvectors is None:
            self.calculate_eigenvalues()
        evs, f, f_inv = self._propagator_factors(number_of_modes)
        if Ts is not None:
            self.Gs = self.transient_growth_gains(Ts, number_of_modes)
        mat = f @ np.diag(np.exp(evs * T)) @ f_inv
        _, s, vh = np.linalg.svd(mat, compute_uv=True)
        coeffs = f_inv @ vh.conj().T[:, 0]
        if save:
            self.S, self.coeffs = s, coeffs
        return s, coeffs

    def calculate_transient_growth_max_energy(self, T: float, number_of_modes: int,
                                              Ts: Optional[List[float]] = None) -> float:
        """Optimal gain S_1^2 at T, reusing the last SVD of the same mode count
        (linear_stability_calculation.py:538-557)."""
        if self.S is None or self.S.shape[0] != min(number_of_modes, len(self.eigenvectors or [])):
            self.S, _ = self.calculate_transient_growth_svd(T, number_of_modes, save=False, Ts=Ts)
        return float(self.S[0] ** 2)

    def calculate_transient_growth_initial_condition_from_coefficients(
            self, domain: PhysicalDomain, coeffs: np.ndarray, recompute: bool = True) -> VectorField:
        """Velocity of sum_k coeffs_k q_k (linear_stability_calculation.py:559-575)."""
        if recompute or self.eigenvectors is None:
            self.calculate_eigenvalues()
        m = len(coeffs)
        combined = np.array(self.eigenvectors[:m]).T @ np.asarray(coeffs)
        return self.velocity_field(domain, combined)

    def calculate_transient_growth_initial_condition(
            self, domain: PhysicalDomain, T: float, number_of_modes: int, recompute_partial: bool = True,
            recompute_full: bool = True, save_final: bool = False, Ts: Optional[List[float]] = None
    ) -> VectorField:
        """The initial velocity that reaches the optimal gain at T
        (linear_stability_calculation.py:577-638)."""
        if recompute_full or self.coeffs is None or self.coeffs.shape[0] != number_of_modes:
            self.S, factors = self.calculate_transient_growth_svd(
                T, number_of_modes, save=False, recompute=recompute_full, Ts=Ts)
        else:
            factors = self.coeffs
        u = self.calculate_transient_growth_initial_condition_from_coefficients(domain, factors, recompute_full)
        if save_final:
            for i in range(len(u)):
                u[i].name = "velocity_perturbation_" + "xyz"[i]
            _no_files("the optimal initial condition")
        return u

    def perform_calculation(self) -> None:
        self.assemble_matrix_fast()
        self.calculate_eigenvalues()


def _no_files(what: str) -> None:
    warnings.warn(f"{what}: file output is not supported, results stay in memory", stacklevel=3)
