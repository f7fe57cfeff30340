"""CPU FP64 oracle for the (v, omega_y) channel-flow step and its dual step.

TEST INFRASTRUCTURE ONLY. This module is a vectorised NumPy restatement of the
reference algorithm (dakling/jax-spectral-dns, package jax_spectral_dns). It is
imported by tests/, by ``__graft_entry__.smoke()`` and by ``bench.py``'s CPU
baseline leg -- always as the checker or the timed CPU baseline, never by the
product path. It is pinned against outputs of the unmodified reference
(tests/golden/*.npz, produced by tests/golden/make_golden.py).

Every function cites the reference code it restates. Conventions are the
reference's: spectral fields are (Mx, Ny, Mz) complex128 (vector fields carry
a leading component axis of 3), kx/kz in FFT order [0..K, -K..-1], y index 0 is
y = +1, coefficients use the ortho FFT of the reference's physical grid divided
by s = Lx Lz / (4 pi^2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# RK3 / Crank-Nicolson coefficients (navier_stokes.py:898-918)
RK_ALPHA = (29 / 96, -3 / 40, 1 / 6)
RK_BETA = (37 / 160, 5 / 24, 1 / 6)
RK_GAMMA = (8 / 15, 5 / 12, 3 / 4)
RK_XI = (0.0, -17 / 60, -5 / 12)


# --------------------------------------------------------------------------
# grid and operators (domain.py)
# --------------------------------------------------------------------------

def cheb_points(n: int) -> np.ndarray:
    """domain.py:130-140 (get_cheb_grid)."""
    return np.array([np.cos(np.pi / (n - 1) * i) for i in np.arange(n)])


def cheb_diff_matrix(xs: np.ndarray) -> np.ndarray:
    """domain.py:155-163 (assemble_cheb_diff_mat, order 1)."""
    n = len(xs)
    c = np.concatenate([[2.0], np.ones(n - 2), [2.0]]) * (-1.0) ** np.arange(n)
    x = np.repeat(xs, n).reshape(n, n)
    dx = x - x.T
    d_ = np.outer(c, 1.0 / c) / (dx + np.eye(n))
    acc = np.zeros(n)
    for j in range(n):  # builtin sum over the rows of d_.T, in index order
        acc = acc + d_[:, j]
    return d_ - np.diag(acc)


def domain_shapes(shape, aliasing=1.5):
    """Mode counts and physical grid sizes of Domain.create (domain.py:201-317)
    for periodic x, Chebyshev y, periodic z."""
    modes, phys = [], []
    for i, n in enumerate(shape):
        n = int(n)
        if i == 1:
            modes.append(n)
            phys.append(n)
            continue
        m = n if n % 2 != 0 else n + 1
        p = math.ceil(m * aliasing)
        p = p if p % 2 != 0 else p + 1
        phys.append(p - 1 if p % 2 != 0 else p)  # get_fourier_grid, domain.py:143-152
        modes.append(m)
    return tuple(modes), tuple(phys)


def fourier_k(m: int, length: float) -> np.ndarray:
    """Wavenumber grid of FourierDomain.FromPhysicalDomain (domain.py:791-848):
    fftshift of linspace(0, M-1, M) minus M//2, times 2 pi / L."""
    inp = np.linspace(0, m - 1, int(m))
    return (np.concatenate([inp[m // 2:], inp[: m // 2]]) - m // 2) * (2 * np.pi) / length


@dataclass
class Grid:
    """Discretisation of one channel box (reference Domain + FourierDomain)."""

    shape: tuple
    lx: float
    lz: float
    aliasing: float = 1.5
    modes: tuple = field(init=False)
    phys: tuple = field(init=False)

    def __post_init__(self):
        self.modes, self.phys = domain_shapes(self.shape, self.aliasing)
        self.mx, self.ny, self.mz = self.modes
        self.px, _, self.pz = self.phys
        self.y = cheb_points(self.ny)
        self.D = cheb_diff_matrix(self.y)
        self.D2 = np.linalg.matrix_power(self.D, 2)
        self.kx = fourier_k(self.mx, self.lx)
        self.kz = fourier_k(self.mz, self.lz)
        self.s = (self.lx / (2 * np.pi)) * (self.lz / (2 * np.pi))
        self.KX = self.kx[:, None, None]
        self.KZ = self.kz[None, None, :]

    # ---- transforms (domain.py:716-764, 1167-1242) -----------------------
    def no_hat(self, f_hat: np.ndarray) -> np.ndarray:
        """field_no_hat: zero-pad [0..K] + zeros + [-K..-1] along x then z,
        ifftn(ortho) over (x, z), real part, times s."""
        out = f_hat
        for ax, m in ((-3, self.mx), (-1, self.mz)):
            k = m // 2
            n_zero = math.ceil(m * (self.aliasing - 1))
            f1 = np.take(out, np.arange(0, k + 1), axis=ax)
            f2 = np.take(out, np.arange(m - k, m), axis=ax)
            zshape = list(f1.shape)
            zshape[ax] = n_zero
            if n_zero == 0:
                f2 = np.take(f2, np.arange(1, f2.shape[ax]), axis=ax)
            out = np.concatenate([f1, np.zeros(zshape), f2], axis=ax)
        return np.fft.ifftn(out, axes=(-3, -1), norm="ortho").real / (1 / self.s)

    def hat(self, f: np.ndarray) -> np.ndarray:
        """field_hat: fftn(ortho)/s, truncate each periodic axis to
        [0..ks-1], ks, conj(ks), [P-ks+1..P-1] (the -K slot holds the
        conjugate of the +K value, per axis in x-then-z order)."""
        out = np.fft.fftn(f, axes=(-3, -1), norm="ortho") / self.s
        for ax, p in ((-3, self.px), (-1, self.pz)):
            ks = int((p - p * (1 - 1 / self.aliasing)) / 2)
            o1 = np.take(out, np.arange(0, ks), axis=ax)
            o2 = np.take(out, np.array([ks]), axis=ax)
            o3 = np.take(out, np.arange(p - ks + 1, p), axis=ax)
            out = np.concatenate([o1, o2, np.conj(o2), o3], axis=ax)
        return out.astype(np.complex128)

    def diff(self, f_hat: np.ndarray, direction: int, order: int = 1) -> np.ndarray:
        """FourierDomain.diff (domain.py:891-918) on (..., Mx, Ny, Mz)."""
        if direction == 0:
            return (1j * self.KX) ** order * f_hat
        if direction == 2:
            return (1j * self.KZ) ** order * f_hat
        return np.einsum("...ijk,lj->...ilk", f_hat, np.linalg.matrix_power(self.D, order))

    def diff_phys_y(self, f: np.ndarray) -> np.ndarray:
        """PhysicalDomain.diff along y (domain.py:355-373)."""
        return np.einsum("...ijk,lj->...ilk", f, self.D)

    def curl(self, v_hat: np.ndarray) -> np.ndarray:
        """FourierDomain.curl (domain.py:920-933)."""
        u_y = self.diff(v_hat[0], 1)
        u_z = self.diff(v_hat[0], 2)
        v_x = self.diff(v_hat[1], 0)
        v_z = self.diff(v_hat[1], 2)
        w_x = self.diff(v_hat[2], 0)
        w_y = self.diff(v_hat[2], 1)
        return np.array([w_y - v_z, u_z - w_x, v_x - u_y])

    def divergence(self, v_hat: np.ndarray) -> np.ndarray:
        """Domain.divergence (domain.py:675-678)."""
        return self.diff(v_hat[0], 0) + self.diff(v_hat[1], 1) + self.diff(v_hat[2], 2)

    # ---- integrals (field.py:1456-1481, 2618-2710; domain.py:485-628) ----
    def y_weights(self) -> np.ndarray:
        """Integration weights: inv(D with first row/col unit) applied to the
        field with its first entry zeroed, value(row 0) - value(row Ny-1)."""
        n = self.ny
        mat = np.block([[np.ones((1, 1)), np.zeros((1, n - 1))], [np.zeros((n - 1, 1)), self.D[1:, 1:]]])
        inv = np.linalg.inv(mat)
        w = inv[0, :] - inv[-1, :]
        w[0] = 0.0
        return w

    def energy(self, v_hat: np.ndarray) -> float:
        """VectorField.no_hat().energy(): sum over components of
        volume_integral(0.5 u^2) / (2 Lx Lz), integrating z, then y, then x."""
        w = self.y_weights()
        total = 0.0
        vol = 2.0 * self.lx * 1.0 * self.lz
        for c in range(v_hat.shape[0]):
            u = self.no_hat(v_hat[c])
            e = 0.5 * u * u
            iz = self.lz / self.pz * e.sum(axis=2)          # (Px, Ny)
            iy = iz @ w                                       # (Px,)
            total += self.lx / self.px * iy.sum() / vol
        return float(total)

    def volume_integral(self, f: np.ndarray) -> float:
        """PhysicalField.volume_integral (field.py:1456-1466): z, then y, then x."""
        iz = self.lz / self.pz * f.sum(axis=2)
        return float(self.lx / self.px * (iz @ self.y_weights()).sum())

    def flow_rate(self, u_hat: np.ndarray) -> float:
        """NavierStokesVelVort.get_flow_rate (navier_stokes.py:709-722):
        y-integral of the streamwise velocity at the grid point x = z = 0."""
        u = self.no_hat(u_hat)
        return float(u[0, :, 0] @ self.y_weights())


def set_bc(f: np.ndarray) -> np.ndarray:
    """update_boundary_conditions (domain.py:630-647): zero the y = +-1 rows."""
    out = f.copy()
    out[..., 0, :] = 0.0
    out[..., -1, :] = 0.0
    return out


# --------------------------------------------------------------------------
# nonlinear terms
# --------------------------------------------------------------------------

def _vel_1_nabla_vel_2(g: Grid, vel_1: np.ndarray, vel_2_hat: np.ndarray) -> np.ndarray:
    """get_vel_1_nabla_vel_2 (navier_stokes.py:76-90): sum_j u1_j d_j u2_i."""
    out = np.zeros_like(vel_1)
    for i in range(3):
        for j in range(3):
            out[i] = out[i] + vel_1[j] * g.no_hat(g.diff(vel_2_hat[i], j))
    return out


def _div_vel_1_vel_2(g: Grid, vel_1_hat: np.ndarray, vel_2: np.ndarray) -> np.ndarray:
    """get_div_vel_1_vel_2 (navier_stokes.py:216-224)."""
    d = g.no_hat(g.divergence(vel_1_hat))
    return np.array([d * vel_2[i] for i in range(3)])


def _helicity_to_nonlinear_terms(g: Grid, hel_hat: np.ndarray, vel_hat: np.ndarray):
    """helicity_to_nonlinear_terms (navier_stokes.py:48-73)."""
    h_v = (-g.diff(g.diff(hel_hat[0], 0) + g.diff(hel_hat[2], 2), 1)
           + g.diff(hel_hat[1], 0, 2) + g.diff(hel_hat[1], 2, 2))
    h_g = g.diff(hel_hat[0], 2) - g.diff(hel_hat[2], 0)
    return h_v, h_g, g.curl(vel_hat), -hel_hat


def nonlinear_ns(g: Grid, vel_hat: np.ndarray):
    """update_nonlinear_terms_high_performance_skew_symmetric
    (navier_stokes.py:236-261): hel = -(u.grad)u + 0.5 (div u) u."""
    vel = np.array([g.no_hat(vel_hat[i]) for i in range(3)])
    div_hat = np.array([g.hat(x) for x in _div_vel_1_vel_2(g, vel_hat, vel)])
    conv = -_vel_1_nabla_vel_2(g, vel, vel_hat)
    hel = np.array([g.hat(conv[i]) for i in range(3)]) + 0.5 * div_hat
    return _helicity_to_nonlinear_terms(g, hel, vel_hat)


def nonlinear_perturbation(g: Grid, vel_hat, base_hat, linearise: bool, coupling_term: bool = True):
    """update_nonlinear_terms_high_performance_perturbation_skew_symmetric
    (navier_stokes_perturbation.py:160-239)."""
    lam = 0.0 if linearise else 1.0
    vel = np.array([g.no_hat(vel_hat[i]) for i in range(3)])
    base = np.array([g.no_hat(base_hat[i]) for i in range(3)])
    div_vv = (lam * _div_vel_1_vel_2(g, vel_hat, vel) + _div_vel_1_vel_2(g, base_hat, vel)
              + _div_vel_1_vel_2(g, vel_hat, base))
    div_hat = np.array([g.hat(div_vv[i]) for i in range(3)])
    # get_helicity_perturbation_convection (navier_stokes_perturbation.py:43-71)
    conv = -(lam * _vel_1_nabla_vel_2(g, vel, vel_hat) + _vel_1_nabla_vel_2(g, base, vel_hat)
             + _vel_1_nabla_vel_2(g, vel, base_hat))
    hel = np.array([g.hat(conv[i]) for i in range(3)]) + 0.5 * div_hat
    h_v, h_g, vort, conv_ns = _helicity_to_nonlinear_terms(g, hel, vel_hat)
    if not coupling_term:
        comb = g.hat(g.diff_phys_y(base[0]) * vel[1])
        h_g = h_g + g.diff(comb, 2)
    return h_v, h_g, vort, conv_ns


def nonlinear_dual(g: Grid, v_hat, base_hat, u_hat, linearise: bool, coupling_term: bool = True):
    """update_nonlinear_terms_high_performance_perturbation_dual_skew_symmetric
    (navier_stokes_perturbation_dual.py:214-294) with re_ijj = 0."""
    v = np.array([g.no_hat(v_hat[i]) for i in range(3)])
    uu_hat = (0.0 if linearise else 1.0) * u_hat + base_hat
    uu = np.array([g.no_hat(uu_hat[i]) for i in range(3)])
    div_vv = 0.5 * (_div_vel_1_vel_2(g, uu_hat, v) + _div_vel_1_vel_2(g, v_hat, uu))
    div_hat = np.array([g.hat(div_vv[i]) for i in range(3)])
    # get_helicity_perturbation_dual_convection (..._dual.py:61-90)
    t1 = _vel_1_nabla_vel_2(g, uu, v_hat)
    t1_hat = np.array([g.hat(t1[i]) for i in range(3)])
    t2_hat = []
    for i in range(3):
        acc = np.zeros_like(v[0])
        for j in range(3):
            acc = acc + v[j] * g.no_hat(g.diff(uu_hat[j], i))
        t2_hat.append(g.hat(acc))
    hel = -t1_hat + np.array(t2_hat) + 0.5 * div_hat
    h_v, h_g, vort, conv_ns = _helicity_to_nonlinear_terms(g, hel, v_hat)
    if not coupling_term:
        comb_hy = g.hat(g.diff_phys_y(g.no_hat(base_hat[0])) * v[0])
        h_v = h_v + g.diff(comb_hy, 0, 2) + g.diff(comb_hy, 2, 2)
    return h_v, h_g, vort, conv_ns


# --------------------------------------------------------------------------
# implicit operators and the RK3/CN step (navier_stokes.py:920-1022, 1219-1775)
# --------------------------------------------------------------------------

def _bc_hom(mat: np.ndarray) -> np.ndarray:
    """enforce_homogeneous_dirichlet (domain.py:375-397)."""
    out = mat.copy()
    out[..., 0, :] = 0.0
    out[..., :, 0] = 0.0
    out[..., 0, 0] = 1.0
    out[..., -1, :] = 0.0
    out[..., :, -1] = 0.0
    out[..., -1, -1] = 1.0
    return out


class Stepper:
    """Restatement of NavierStokesVelVort.perform_runge_kutta_step with the
    per-wavenumber operators of prepare_assemble_rk_matrices and
    assemble_poisson_matrix, batched over wavenumber pairs that share
    kx^2 + kz^2 (their matrices are identical in the reference too).

    kind: "ns" (full Navier-Stokes), "perturbation" or "dual".
    dt is the step used by the implicit operators; dt_explicit multiplies the
    explicit terms (the dual re-uses the forward operators with dt negated in
    the explicit part, navier_stokes_perturbation_dual.py:470-471, 571-587).
    """

    def __init__(self, g: Grid, re_tau: float, dt: float, kind: str = "ns",
                 constant_mass_flux: bool = False, linearise: bool = False,
                 coupling_term: bool = True, base_hat=None, dt_explicit=None,
                 flow_rate_target: float = 0.0):
        self.g, self.re_tau, self.dt, self.kind = g, re_tau, dt, kind
        self.dt_explicit = dt if dt_explicit is None else dt_explicit
        self.cmf = constant_mass_flux
        self.linearise = linearise
        self.coupling_term = coupling_term
        self.base_hat = base_hat
        self.flow_rate_target = flow_rate_target
        self.u_history = None  # dual: callable t -> forward state
        self.source = None  # callable t -> (3, Mx, Ny, Mz) source or None (get_source_term)
        # time-dependent base flow t -> base_hat (NavierStokesVelVortPerturbationInstationary);
        # linearise / coupling_term may also be callables t -> bool (the *_switch parameters)
        self.base_fn = None
        self._prepare()

    def _prepare(self):
        g, n = self.g, self.g.ny
        ax = np.abs(np.round(g.kx * g.lx / (2 * np.pi))).astype(int)
        az = np.abs(np.round(g.kz * g.lz / (2 * np.pi))).astype(int)
        kxu = np.arange(ax.max() + 1) * (2 * np.pi) / g.lx
        kzu = np.arange(az.max() + 1) * (2 * np.pi) / g.lz
        nux, nuz = len(kxu), len(kzu)
        self.uidx = ax[:, None] * nuz + az[None, :]          # (Mx, Mz) -> unique id
        ksq = (kxu[:, None] ** 2 + kzu[None, :] ** 2).reshape(-1)
        self.ksq = ksq
        # groups of (xi, zi) sharing a unique id (at most 4: +-kx, +-kz)
        nu = nux * nuz
        gx = np.zeros((nu, 4), dtype=int)
        gz = np.zeros((nu, 4), dtype=int)
        cnt = np.zeros(nu, dtype=int)
        for xi in range(g.mx):
            for zi in range(g.mz):
                u = self.uidx[xi, zi]
                gx[u, cnt[u]] = xi
                gz[u, cnt[u]] = zi
                cnt[u] += 1
        for u in range(nu):
            for c in range(cnt[u], 4):
                gx[u, c], gz[u, c] = gx[u, 0], gz[u, 0]
        self.gx, self.gz = gx, gz

        eye = np.eye(n)
        Ly = 1 / self.re_tau * g.D2
        eye_bc = np.zeros((n, n))
        eye_bc[1:-1, 1:-1] = np.eye(n - 2)
        D2_hom = _bc_hom(g.D2)
        self.lhs_inv = []
        self.rhs = []
        self.va = []
        self.minv = []
        # assemble_poisson_matrix (domain.py:857-889)
        self.poisson = np.linalg.inv(-ksq[:, None, None] * eye_bc[None] + D2_hom[None])
        for st in range(3):
            L = Ly[None] + eye[None] * (-ksq[:, None, None]) / self.re_tau
            rhs = _bc_hom(eye[None] + RK_ALPHA[st] * self.dt * L)
            lhs = _bc_hom(eye[None] - RK_BETA[st] * self.dt * L)
            self.rhs.append(rhs)
            self.lhs_inv.append(np.linalg.inv(lhs))
            # inhomogeneous problem (enforce_inhomogeneous_dirichlet, domain.py:425-448)
            lhs_in = eye[None] - RK_BETA[st] * self.dt * L
            lhs_in[:, 0, :] = 0.0
            lhs_in[:, 0, 0] = 1.0
            lhs_in[:, -1, :] = 0.0
            lhs_in[:, -1, -1] = 1.0
            rhs_in = np.zeros(n)
            rhs_in[0] = 1.0  # bc_right = 1 sits at y = +1
            phi_a = np.linalg.inv(lhs_in) @ rhs_in
            va = np.einsum("uij,uj->ui", self.poisson, phi_a)
            va[:, 0] = 0.0
            va[:, -1] = 0.0
            vb = va[:, ::-1]
            dva = va @ g.D.T
            dvb = vb @ g.D.T
            M = np.stack([np.stack([dva[:, 0], dvb[:, 0]], -1), np.stack([dva[:, -1], dvb[:, -1]], -1)], -2)
            self.va.append(va)
            self.minv.append(np.linalg.inv(M))
        # (0,0) mean-flow block system (navier_stokes.py:1000-1022)
        Z = np.zeros((n, n))
        L_ns = 1 / self.re_tau * np.block([[D2_hom, Z], [Z, D2_hom]])
        I_ns = np.eye(2 * n)
        self.rhs_ns, self.lhs_inv_ns = [], []
        for st in range(3):
            self.rhs_ns.append(_bc_hom(I_ns + RK_ALPHA[st] * self.dt * L_ns))
            self.lhs_inv_ns.append(np.linalg.inv(_bc_hom(I_ns - RK_BETA[st] * self.dt * L_ns)))

    # --- per-wavenumber batched matrix application -----------------------
    def _apply(self, mats: np.ndarray, X: np.ndarray) -> np.ndarray:
        """out[kx, :, kz] = mats[uid(kx,kz)] @ X[kx, :, kz] for complex X."""
        xg = X[self.gx, :, self.gz]                     # (nu, 4, Ny)
        xr = np.ascontiguousarray(np.moveaxis(xg, 1, 2)).view(np.float64)  # (nu, Ny, 8)
        yr = np.matmul(mats, xr)
        yg = np.moveaxis(yr.view(np.complex128), 2, 1)  # (nu, 4, Ny)
        out = np.empty_like(X)
        out[self.gx, :, self.gz] = yg
        return out

    def _nonlinear(self, vel_hat, t):
        g = self.g
        lin = self.linearise(t) if callable(self.linearise) else self.linearise
        cpl = self.coupling_term(t) if callable(self.coupling_term) else self.coupling_term
        base = self.base_fn(t) if self.base_fn is not None else self.base_hat
        if self.kind == "ns":
            return nonlinear_ns(g, vel_hat)
        if self.kind == "perturbation":
            return nonlinear_perturbation(g, vel_hat, base, lin, cpl)
        return nonlinear_dual(g, vel_hat, base, self.u_history(t), lin, cpl)

    def rk_step(self, vel_hat: np.ndarray, dpdx: float, time_step: int):
        """perform_runge_kutta_step + enforce_constant_mass_flux
        (navier_stokes.py:1219-1775, 1205-1214)."""
        g = self.g
        dt_e = self.dt_explicit
        hv_old = hg_old = conv_old = None
        src = self.source(time_step) if self.source is not None else None
        for st in range(3):
            h_v, h_g, vort, conv = self._nonlinear(vel_hat, time_step)
            if src is not None:
                # navier_stokes.py:1697-1703, indexing as written there: the y
                # component C of curl(source) is (Mx, Ny, Mz); C[0], C[2] are
                # its kx index 0 and 2 planes, whose x/z derivatives broadcast
                # over kx before [1] picks the kx index 1 plane again
                C = g.curl(src)[1]
                h_v = h_v + (1j * g.KZ * C[0][None] - 1j * g.KX * C[2][None])[1][None]
                h_g = h_g + C[1][None]
            if st == 0:
                hv_old = np.zeros_like(h_v)
                hg_old = np.zeros_like(h_g)
                conv_old = np.zeros_like(conv)
            v1 = vel_hat[1]
            phi = g.diff(v1, 0, 2) + g.diff(v1, 1, 2) + g.diff(v1, 2, 2)
            # v: p-part
            rhs_p = self._apply(self.rhs[st], phi) + (dt_e * RK_GAMMA[st]) * h_v + (dt_e * RK_XI[st]) * hv_old
            rhs_p = set_bc(rhs_p)
            phi_new = set_bc(self._apply(self.lhs_inv[st], rhs_p))
            v_p = set_bc(self._apply(self.poisson, phi_new))
            # a/b-parts and the influence-matrix correction (lstsq of a 2x2)
            va = self.va[st][self.uidx]                       # (Mx, Mz, Ny)
            va = np.moveaxis(va, 2, 1)                        # (Mx, Ny, Mz)
            vb = va[:, ::-1, :]
            dvp = np.einsum("lj,ijk->ilk", g.D[[0, -1]], v_p)  # (Mx, 2, Mz)
            R = -dvp
            minv = self.minv[st][self.uidx]                   # (Mx, Mz, 2, 2)
            ab = np.einsum("xzij,xjz->xiz", minv, R)
            v_new = set_bc(v_p + ab[:, 0:1, :] * va + ab[:, 1:2, :] * vb)
            # omega_y
            rhs_w = self._apply(self.rhs[st], vort[1]) + (dt_e * RK_GAMMA[st]) * h_g + (dt_e * RK_XI[st]) * hg_old
            om_new = set_bc(self._apply(self.lhs_inv[st], set_bc(rhs_w)))
            # u, w from continuity (rk_not_00)
            vy = np.einsum("ijk,lj->ilk", v_new, g.D)
            k2 = -(g.KX ** 2 + g.KZ ** 2)
            k2s = np.where(k2 == 0, 1.0, k2)
            u_new = (-1j * g.KX * vy + 1j * g.KZ * om_new) / k2s
            w_new = (-1j * g.KZ * vy - 1j * g.KX * om_new) / k2s
            # (0,0) mean flow (rk_00)
            u00, w00 = self._mean_flow(st, vel_hat, conv, conv_old, dpdx, time_step, src)
            u_new[0, :, 0] = u00
            w_new[0, :, 0] = w00
            hv_old, hg_old, conv_old = h_v, h_g, conv
            vel_hat = set_bc(np.array([u_new, v_new, w_new]))
        return self._mass_flux(vel_hat, dpdx)

    def _mean_flow(self, st, vel_hat, conv, conv_old, dpdx, time_step, source=None):
        g, n = self.g, self.g.ny
        v_hat = np.concatenate([vel_hat[0][0, :, 0], vel_hat[2][0, :, 0]])
        scale = ((g.px * (2 * np.pi / g.lx) ** 2) * (g.pz * (2 * np.pi / g.lz) ** 2)) ** 0.5
        dp = dpdx * scale
        src = np.concatenate([-dp * np.ones(n), np.zeros(n)])
        if source is not None:  # navier_stokes.py:1461-1491
            src = src + np.concatenate([source[0][0, :, 0], source[2][0, :, 0]])
        N_new = np.concatenate([-conv[0][0, :, 0], -conv[2][0, :, 0]]) + src
        N_old = np.concatenate([-conv_old[0][0, :, 0], -conv_old[2][0, :, 0]]) + src
        out = self.lhs_inv_ns[st] @ (self.rhs_ns[st] @ v_hat + (self.dt_explicit * RK_GAMMA[st]) * N_new
                                     + (self.dt_explicit * RK_XI[st]) * N_old)
        return out[:n], out[n:]

    def _mass_flux(self, vel_hat, dpdx):
        """enforce_constant_mass_flux: dPdx += (Q - Q0)/dt, u += -(Q - Q0)/2
        through a no_hat/hat round trip (navier_stokes.py:724-805;
        perturbation variant with Q0 = 0, navier_stokes_perturbation.py:420-466)."""
        if not self.cmf:
            return vel_hat, dpdx
        g = self.g
        q = g.flow_rate(vel_hat[0])
        diff = q - self.flow_rate_target
        dpdx = dpdx + diff / self.dt_explicit
        u = g.no_hat(vel_hat[0]) + np.ones((g.px, g.ny, g.pz)) * (-1 * diff * 0.5)
        out = vel_hat.copy()
        out[0] = g.hat(u)
        return out, dpdx


# --------------------------------------------------------------------------
# equation-level drivers
# --------------------------------------------------------------------------

def make_stepper(kind: str, shape, lx, lz, re_tau, dt, **kw) -> Stepper:
    g = Grid(tuple(shape), lx, lz)
    if kind in ("perturbation", "dual") and kw.get("base_hat") is None:
        kw["base_hat"] = laminar_base_hat(g, kw.pop("u_max", 1.0))
    return Stepper(g, re_tau, dt, kind=kind, **kw)


def laminar_base_hat(g: Grid, u_max: float = 1.0) -> np.ndarray:
    """Default base flow u_max (1 - y^2) built as the reference builds it:
    PhysicalField.FromFunc(...).hat() (navier_stokes_perturbation.py:351-380)."""
    X = np.meshgrid(np.zeros(g.px), g.y, np.zeros(g.pz), indexing="ij")[1]
    ux = u_max * (1 - X ** 2)
    zero = 0.0 * X
    return np.array([g.hat(ux), g.hat(zero), g.hat(zero)])


def instationary_base_hat(g: Grid, t: float, re: float, kappa: float = 1.0, accelerate: bool = True,
                          n_max: int = 100) -> np.ndarray:
    """Base flow of NavierStokesVelVortPerturbationInstationary.vel_base_fn
    (navier_stokes_perturbation_instationary.py:37-83) at time t: wall-driven
    profile with wall speed g_w(t) = 1 - exp(-kappa t) (accelerate) or
    exp(-kappa t) and its series correction, built on the physical grid and
    transformed like the reference."""
    gw = (1.0 - np.exp(-kappa * t)) if accelerate else np.exp(-kappa * t)
    dgw = (kappa * np.exp(-kappa * t)) if accelerate else (-kappa * np.exp(-kappa * t))
    dgw0 = kappa if accelerate else -kappa
    y = g.y
    prof = gw * y + re / 6 * dgw * (y ** 3 - y)
    coeff = -1.0 if accelerate else 1.0
    for n in range(1, n_max):
        c1n = (-2 * re * (-1) ** n / (np.pi * n) ** 3) * dgw0
        a_n = (np.pi * n) ** 2 / re
        integ = kappa ** 2 * coeff / (a_n - kappa)
        prof = prof + (np.exp(-kappa * t) - np.exp(-a_n * t)) * (
            -(2 * re * (-1) ** n) / (np.pi * n) ** 3 * integ * np.sin(n * np.pi * y))
        prof = prof + np.exp(-a_n * t) * c1n * np.sin(n * np.pi * y)
    ux = np.broadcast_to(prof[None, :, None], (g.px, g.ny, g.pz)).copy()
    zero = np.zeros_like(ux)
    return np.array([g.hat(ux), g.hat(zero), g.hat(zero)])


def run(stepper: Stepper, u0: np.ndarray, n_steps: int, dpdx: float = 0.0, history: bool = False):
    """Advance n_steps; returns the final state, dPdx and optionally the states
    u_0..u_n (the write_entire_output trajectory of solve_scan)."""
    u = u0.copy()
    hist = [u] if history else None
    for t in range(n_steps):
        u, dpdx = stepper.rk_step(u, dpdx, t)
        if history:
            hist.append(u)
    return u, dpdx, hist


def dissipation_average(g: Grid, hist, re_tau: float) -> float:
    """get_dissipation_average (navier_stokes_perturbation_dual.py:1089-1104):
    sum over the stored states of sum_ij (d_j u_i)^2, squares of the spectral
    coefficients, over |Re_tau n|, then no_hat and the volume integral. The x-z
    integral leaves the (0, 0) mode of that sum."""
    acc = np.zeros(hist[0].shape[1:], dtype=complex)
    for u in hist:
        for i in range(3):
            for j in range(3):
                acc += g.diff(u[i], j) ** 2
    acc /= abs(re_tau * len(hist))
    return float(g.volume_integral(g.no_hat(acc)))


def dissipation_gradient(shape, lx, lz, re, dt, n_steps, u0, linearise, u_max=1.0):
    """The dual's dissipation objective (navier_stokes_perturbation_dual.py:
    904-990, 1089-1120): the dual starts from zero and every step t adds the
    source -lap(u(T - t)) / |Re_tau T| of the forward state it pairs with;
    grad = (u0 - v0) / E0. Returns (grad, value, v0)."""
    re_tau = re / u_max
    fwd = make_stepper("perturbation", shape, lx, lz, re_tau, dt, linearise=linearise, u_max=u_max)
    _, _, hist = run(fwd, u0, n_steps, history=True)
    g = fwd.g
    dual = Stepper(g, re_tau, dt, kind="dual", linearise=linearise, base_hat=fwd.base_hat, dt_explicit=-dt)
    dual.u_history = lambda t: hist[-1 - t]
    end_time = n_steps * dt

    def source(t):
        u = hist[-1 - t]
        lap = np.array([g.diff(u[i], 0, 2) + g.diff(u[i], 1, 2) + g.diff(u[i], 2, 2) for i in range(3)])
        return -1.0 / abs(re_tau * end_time) * lap

    dual.source = source
    v0, _, _ = run(dual, np.zeros_like(u0), n_steps)
    return (u0 - v0) / g.energy(u0), dissipation_average(g, hist, re_tau), v0


def dual_gradient(shape, lx, lz, re, dt, n_steps, u0, linearise, u_max=1.0):
    """NavierStokesVelVortPerturbationDual.get_grad for the 'gain' objective
    (navier_stokes_perturbation_dual.py:850-939, 1037-1120): forward run with
    the full trajectory, dual run from -u(T) with Re and dt negated (implicit
    operators from the forward equation), grad = (u0 - v0) / E0."""
    re_tau = re / u_max
    fwd = make_stepper("perturbation", shape, lx, lz, re_tau, dt, linearise=linearise, u_max=u_max)
    uT, _, hist = run(fwd, u0, n_steps, history=True)
    dual = Stepper(fwd.g, re_tau, dt, kind="dual", linearise=linearise,
                   base_hat=fwd.base_hat, dt_explicit=-dt)
    dual.u_history = lambda t: hist[-1 - t]
    v0, _, _ = run(dual, -uT, n_steps)
    e0 = fwd.g.energy(u0)
    gain = fwd.g.energy(uT) / e0
    return (u0 - v0) / e0, gain, v0, uT
