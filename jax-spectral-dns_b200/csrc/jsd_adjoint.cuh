// Discrete adjoint of the linearised perturbation step: the exact transpose
// (for the real inner product of the interleaved real and imaginary parts) of
// the map one RK3/Crank-Nicolson step applies to a state, kernel by kernel in
// reverse order. The forward stage, as the step kernels compute it in exact
// arithmetic (navier_stokes.py:1228-1548 and navier_stokes_perturbation.py:
// 160-239 with lambda = 0):
//   1  dv = D v
//   2  P = linear terms of (u, v, w, dv) at the source modes, h = RT(P)
//      (Hermitian part, then the reference's truncation quirk)
//   3  q = i kx h0 + i kz h2, H1 = h1, hg = i kz h0 - i kx h2, conv00 = -(h0, h2)(0,0)
//   4  omega = i kz u - i kx w
//   5  X1 = V^-1 D q, T0 = V^-1 H1, T1 = V^-1 hg, vt = V^-1 v, omt = V^-1 omega
//   6  per column: diagonal solves and influence-matrix correction (k_eigen_update)
//   7  (0,0): x00_new = LR x00 + Linv dt_e (gamma N + xi N_old), N = -conv00
//   8  v = V vn, dvn = D V vn, om = V omn
//   9  u, w from continuity, (0,0) from x00_new, walls zeroed (k_reconstruct)
// The adjoint runs 9' .. 1' with the transposed operators; the terms a stage
// hands to the next one (h_v, h_g of step 6 and conv00) carry their
// cotangents backwards between stages. The carried quantities of the forward
// step (V^-1 v, omega_y and dv/dy of the new state) are mathematically the
// ones recomputed here, so the transpose is that of the computed map up to
// round-off.
#pragma once

#include "jsd_common.cuh"
#include "jsd_spectral.cuh"

namespace jsd {

// 9'. Cotangent (lu, lw) of the new state's u, w -> cotangents of dv/dy,
// omega_y (non-(0,0) modes, interior rows) and of the mean-flow solution
// (x00: u00 then w00 per Chebyshev point; zero at the walls, which the forward
// step overwrites).
__global__ void k_reconstruct_adj(Geo g, const double2* __restrict__ lu, const double2* __restrict__ lw,
                                  double2* __restrict__ dv_bar, double2* __restrict__ om_bar,
                                  double2* __restrict__ x00_bar) {
  const size_t total = (size_t)g.ny * g.nk;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(t / g.nk);
    const int r = (int)(t - (size_t)y * g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    const bool wall = (y == 0 || y == g.ny - 1);
    if (ix == 0 && iz == 0) {
      dv_bar[t] = om_bar[t] = make_double2(0.0, 0.0);
      x00_bar[y] = wall ? make_double2(0.0, 0.0) : lu[t];
      x00_bar[g.ny + y] = wall ? make_double2(0.0, 0.0) : lw[t];
      continue;
    }
    if (wall) {
      dv_bar[t] = om_bar[t] = make_double2(0.0, 0.0);
      continue;
    }
    const double kx = kx_of(g, ix), kz = kz_of(g, iz);
    const double ik2 = 1.0 / (kx * kx + kz * kz);
    const double2 a = lu[t], b = lw[t];
    // u = i kx / k^2 dv - i kz / k^2 om, w = i kz / k^2 dv + i kx / k^2 om: conjugate coefficients
    dv_bar[t] = cscale(cadd(cmul_ik(a, -kx), cmul_ik(b, -kz)), ik2);
    om_bar[t] = cscale(csub(cmul_ik(a, kz), cmul_ik(b, kx)), ik2);
  }
}

// 6'. Transpose of k_eigen_update for one stage, one thread per real column
// (same block shape as the forward kernel). Inputs: the cotangents of the new
// V^-1 v (two parts, summed: from v and from dv/dy) and of the new V^-1
// omega_y, and in hv_old / hg_old the cotangents of this stage's h_v~, h_g~
// terms as the next stage read them (ignored when `last`: the next step's first
// stage does not read them). Outputs: cotangents of X1, T0 (= V^-1 H1), T1
// (= V^-1 h_g), V^-1 v, V^-1 omega_y; of the wall values v(+1), v(-1) (rows 0
// and ny-1 of wall_out, a spectral field whose interior rows the caller fills
// later); and in hv_old / hg_old the cotangents of the previous stage's terms.
__global__ void __launch_bounds__(kEigCols * kEigParts, 4) k_eigen_update_adj(
    Geo g, EigTables t, StageCoef sc, int last, const double* __restrict__ vn_bar_a,
    const double* __restrict__ vn_bar_b, const double* __restrict__ omn_bar, double* __restrict__ hv_old,
    double* __restrict__ hg_old, double* __restrict__ X1_bar, double* __restrict__ T0_bar,
    double* __restrict__ T1_bar, double* __restrict__ vt_bar, double* __restrict__ omt_bar,
    double* __restrict__ wall_out) {
  __shared__ double red[kEigParts][4][kEigCols];
  const int N = 2 * g.nk;
  const int lane = threadIdx.x % kEigCols;
  const int part = threadIdx.x / kEigCols;
  const int c = blockIdx.x * kEigCols + lane;
  const bool active = c < N;
  const int n = g.ny - 2;
  const int j0 = (n * part) / kEigParts, j1 = (n * (part + 1)) / kEigParts;
  double k2 = 0.0;
  if (active) {
    const int kp = c >> 1;
    const int ix = kp / g.mz, iz = kp - (kp / g.mz) * g.mz;
    const double kx = kx_of(g, ix), kz = kz_of(g, iz);
    k2 = kx * kx + kz * kz;
  }
  const double ar = sc.alpha * sc.dt / sc.re;
  const double br = sc.beta * sc.dt / sc.re;
  // influence-matrix sums: the forward's (d0a, dNa, d0b, dNb) and the adjoint's (a_bar, b_bar)
  double d0a = 0, dNa = 0, d0b = 0, dNb = 0, abar = 0, bbar = 0;
  if (active) {
    for (int j = j0; j < j1; ++j) {
      const size_t o = (size_t)j * N + c;
      const double L = t.lam[j] - k2;
      const double H = 1.0 - br * L;
      const double va = br * t.c0[j] / (H * L);
      const double sg = t.sgn[j];
      d0a += t.w0[j] * va;
      dNa += t.wN[j] * va;
      d0b += t.w0[j] * sg * va;
      dNb += t.wN[j] * sg * va;
      const double vnb = vn_bar_a[o] + vn_bar_b[o];
      abar += vnb * va;
      bbar += vnb * sg * va;
    }
  }
  red[part][0][lane] = d0a;
  red[part][1][lane] = dNa;
  red[part][2][lane] = abar;
  red[part][3][lane] = bbar;
  // (d0b, dNb) are sgn-weighted copies of (d0a, dNa) per row; reduce them too
  __shared__ double red2[kEigParts][2][kEigCols];
  red2[part][0][lane] = d0b;
  red2[part][1][lane] = dNb;
  __syncthreads();
  double w0sum = 0.0, wNsum = 0.0;  // cotangents of v(+1), v(-1) through phi
  if (active) {
    double s[4] = {0, 0, 0, 0}, s2[2] = {0, 0};
#pragma unroll
    for (int pp = 0; pp < kEigParts; ++pp) {
#pragma unroll
      for (int q = 0; q < 4; ++q) s[q] += red[pp][q][lane];
      s2[0] += red2[pp][0][lane];
      s2[1] += red2[pp][1][lane];
    }
    // forward: sum = (d0p, dNp, d0a, dNa, d0b, dNb); a = (-s5 d0p + s4 dNp)/det,
    // b = (s3 d0p - s2 dNp)/det with det = s2 s5 - s4 s3 (indices of the forward's sum[])
    const double S2 = s[0], S3 = s[1], S4 = s2[0], S5 = s2[1];
    const double det = S2 * S5 - S4 * S3;
    const double abar_ = s[2], bbar_ = s[3];
    const double d0p_bar = (-S5 * abar_ + S3 * bbar_) / det;
    const double dNp_bar = (S4 * abar_ - S2 * bbar_) / det;
    for (int j = j0; j < j1; ++j) {
      const size_t o = (size_t)j * N + c;
      const double L = t.lam[j] - k2;
      const double R = 1.0 + ar * L;
      const double H = 1.0 - br * L;
      const double ih = 1.0 / H;
      const double ihl = ih / L;
      const double vpb = vn_bar_a[o] + vn_bar_b[o] + t.w0[j] * d0p_bar + t.wN[j] * dNp_bar;
      const double phib = R * ihl * vpb;
      const double hvb = sc.dt_e * sc.gamma * ihl * vpb + (last ? 0.0 : hv_old[o]);
      const double ob = omn_bar[o];
      const double hgb = sc.dt_e * sc.gamma * ih * ob + (last ? 0.0 : hg_old[o]);
      vt_bar[o] = L * phib;
      w0sum += t.c0[j] * phib;
      wNsum += t.cN[j] * phib;
      X1_bar[o] = -hvb;
      T0_bar[o] = -k2 * hvb;
      T1_bar[o] = hgb;
      omt_bar[o] = R * ih * ob;
      hv_old[o] = sc.dt_e * sc.xi * ihl * vpb;
      hg_old[o] = sc.dt_e * sc.xi * ih * ob;
    }
  }
  // wall cotangents: sum over the parts of this column, fixed order
  __syncthreads();
  red2[part][0][lane] = w0sum;
  red2[part][1][lane] = wNsum;
  __syncthreads();
  if (active && part == 0) {
    double a0 = 0.0, aN = 0.0;
#pragma unroll
    for (int pp = 0; pp < kEigParts; ++pp) {
      a0 += red2[pp][0][lane];
      aN += red2[pp][1][lane];
    }
    wall_out[c] = a0;
    wall_out[(size_t)(g.ny - 1) * N + c] = aN;
  }
}

// 7'. Transpose of the (0,0) mean-flow update of stage s: x00_bar <- LR^T
// ubar, f_bar = Linv^T ubar; conv_bar (this stage) -= dt_e gamma f_bar,
// conv_bar_prev -= dt_e xi f_bar (null for the first stage). lrT / liT are the
// stage's transposed matrices (2 Ny x 2 Ny, row-major). One warp per row of
// the transposed product.
__global__ void __launch_bounds__(32 * kMeanFlowRows) k_mean_flow_adj(
    Geo g, const double* __restrict__ lrT, const double* __restrict__ liT, const double2* __restrict__ ubar,
    double dt_gamma, double dt_xi, double2* __restrict__ x00_out, double2* __restrict__ conv_bar,
    double2* __restrict__ conv_bar_prev) {
  const int n2 = 2 * g.ny;
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kMeanFlowRows + (threadIdx.x >> 5);
  if (i >= n2) return;
  const double* lr = lrT + (size_t)i * n2;
  const double* li = liT + (size_t)i * n2;
  double ax = 0.0, ay = 0.0, fx = 0.0, fy = 0.0;
  for (int j = lane; j < n2; j += 32) {
    const double2 b = ubar[j];
    ax += lr[j] * b.x;
    ay += lr[j] * b.y;
    fx += li[j] * b.x;
    fy += li[j] * b.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
    fx += __shfl_down_sync(0xffffffffu, fx, o);
    fy += __shfl_down_sync(0xffffffffu, fy, o);
  }
  if (lane == 0) {
    x00_out[i] = make_double2(ax, ay);
    conv_bar[i] = csub(conv_bar[i], make_double2(dt_gamma * fx, dt_gamma * fy));
    if (conv_bar_prev) conv_bar_prev[i] = csub(conv_bar_prev[i], make_double2(dt_xi * fx, dt_xi * fy));
  }
}

// Cotangent of the terms (h0, h1, h2) at output slot (y, ix, iz) from the
// cotangents of q, H1, h_g (interior rows for H1, h_g) and of conv00.
__device__ __forceinline__ void terms_bar(const Geo& g, int y, int ix, int iz, const double2* __restrict__ qb,
                                          const double2* __restrict__ H1b, const double2* __restrict__ hgb,
                                          const double2* __restrict__ convb, double2* hb) {
  const double kx = kx_of(g, ix), kz = kz_of(g, iz);
  const size_t o = sidx(g, y, ix, iz);
  const bool wall = (y == 0 || y == g.ny - 1);
  const double2 q = qb[o];
  const double2 hg = wall ? make_double2(0.0, 0.0) : hgb[o];
  // q = i kx h0 + i kz h2, hg = i kz h0 - i kx h2, conv00 = -(h0, h2)
  hb[0] = cadd(cmul_ik(q, -kx), cmul_ik(hg, -kz));
  hb[1] = wall ? make_double2(0.0, 0.0) : H1b[o];
  hb[2] = csub(cmul_ik(hg, kx), cmul_ik(q, kz));
  if (ix == 0 && iz == 0) {
    hb[0] = csub(hb[0], convb[y]);
    hb[2] = csub(hb[2], convb[g.ny + y]);
  }
}

// 4' .. 2' plus the assembly of the state cotangent: thread per input slot
// p = (y, signed mode (px, pz)). The forward slot t reads the source modes
// (sx, sz) and (-sx, -sz) (truncation_source) with the Hermitian part
// s = (P(sx, sz) + conj P(-sx, -sz)) / 2 and conjugates when the quirk says
// so; slot p is the first source of the slots t whose (sx, sz) = p and the
// second source of those with (sx, sz) = -p. A mode +K is the source of the
// slots +K and -K of its axis; -K is nobody's first source.
// Writes the cotangents of u, w and of v (all but D^T dv_bar, added later) of
// the stage's input state, and dv_bar (cotangent of dv = D v).
__device__ __forceinline__ int sources_of(const Geo& g, int pm, int kmax, int m, int* out) {
  // output positions ix whose truncation source along this axis is the signed mode pm
  if (pm == kmax) {
    out[0] = kmax;
    out[1] = kmax + 1;
    return 2;
  }
  if (pm == -kmax) return 0;
  out[0] = mode_pos(pm, m);
  return 1;
}

__global__ void k_linear_terms_adj(Geo g, const double* __restrict__ ubase, const double* __restrict__ dubase,
                                   const double2* __restrict__ qb, const double2* __restrict__ H1b,
                                   const double2* __restrict__ hgb, const double2* __restrict__ convb,
                                   const double2* __restrict__ omb, const double2* __restrict__ vextra,
                                   const double2* __restrict__ x00, double2* __restrict__ lu,
                                   double2* __restrict__ lv, double2* __restrict__ lw, double2* __restrict__ dvb) {
  const size_t total = (size_t)g.ny * g.nk;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(t / g.nk);
    const int r = (int)(t - (size_t)y * g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    const int px = signed_mode(ix, g.mx), pz = signed_mode(iz, g.mz);
    double2 Pb[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int pass = 0; pass < 2; ++pass) {
      // pass 0: slots whose first source is p; pass 1: slots whose second source is p
      const int sxm = pass == 0 ? px : -px, szm = pass == 0 ? pz : -pz;
      int xs[2], zs[2];
      const int nx = sources_of(g, sxm, g.kx_max, g.mx, xs);
      const int nz = sources_of(g, szm, g.kz_max, g.mz, zs);
      for (int a = 0; a < nx; ++a)
        for (int bb = 0; bb < nz; ++bb) {
          const int ox = xs[a], oz = zs[bb];
          int sx, sz;
          bool cj;
          truncation_source(g, ox, oz, sx, sz, cj);
          double2 hb[3];
          terms_bar(g, y, ox, oz, qb, H1b, hgb, convb, hb);
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const double2 s = cj ? cconj(hb[f]) : hb[f];
            const double2 c = pass == 0 ? s : cconj(s);
            Pb[f] = cadd(Pb[f], cscale(c, 0.5));
          }
        }
    }
    // transpose of linear_pre<kPerturbation> at mode p:
    //   P0 = -ub/2 i kx u - dub v + ub/2 dv + ub/2 i kz w, P1 = -ub i kx v, P2 = -ub i kx w
    const double kx = px * g.ax, kz = pz * g.az;
    const double ub = ubase[y], dub = dubase[y];
    double2 bu = cscale(cmul_ik(Pb[0], kx), 0.5 * ub);
    double2 bv = csub(cscale(cmul_ik(Pb[1], kx), ub), cscale(Pb[0], dub));
    double2 bw = cadd(cscale(cmul_ik(Pb[0], -kz), 0.5 * ub), cscale(cmul_ik(Pb[2], kx), ub));
    const double2 bdv = cscale(Pb[0], 0.5 * ub);
    // omega = i kz u - i kx w (interior rows of omega_bar)
    if (y > 0 && y < g.ny - 1) {
      const double2 ob = omb[t];
      bu = cadd(bu, cmul_ik(ob, -kz));
      bw = cadd(bw, cmul_ik(ob, kx));
    }
    // V^-1 v (interior) and the wall values, from the eigenbasis transpose
    bv = cadd(bv, vextra[t]);
    // (0,0): the mean-flow input x00 = (u00, w00) at every Chebyshev point
    if (ix == 0 && iz == 0) {
      bu = cadd(bu, x00[y]);
      bw = cadd(bw, x00[g.ny + y]);
    }
    lu[t] = bu;
    lv[t] = bv;
    lw[t] = bw;
    dvb[t] = bdv;
  }
}

__global__ void k_add_field(size_t n, const double2* __restrict__ a, double2* __restrict__ out) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    out[t] = cadd(out[t], a[t]);
}

// Gradient of the kinetic energy (k_plane_sums / k_weighted_total: E = s
// sum_y w_y sum |Sym f|^2 over the three components, s = c_inv^2 / 4) with
// respect to the real and imaginary parts of every coefficient: 2 s w_y Sym f
// (Sym, the Hermitian part, is an orthogonal projection).
__global__ void k_energy_grad(Geo g, const double2* __restrict__ f, const double* __restrict__ w, double scale2,
                              double2* __restrict__ out) {
  const size_t fs = (size_t)g.ny * g.nk;
  const size_t total = 3 * fs;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(t / fs);
    const size_t tt = t - (size_t)c * fs;
    const int y = (int)(tt / g.nk);
    const int r = (int)(tt - (size_t)y * g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    const double2 s = sym_at(g, f + c * fs, y, signed_mode(ix, g.mx), signed_mode(iz, g.mz));
    out[t] = cscale(s, scale2 * w[y]);
  }
}

}  // namespace jsd
