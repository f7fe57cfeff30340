// Spectral-space kernels of the RK3/Crank-Nicolson velocity-vorticity step.
//
// Nonlinear terms (skew-symmetric form, reference navier_stokes.py:236-261 and
// navier_stokes_perturbation.py:160-239) are evaluated pseudo-spectrally in
// three fused passes over the y-planes:
//   k_zinv : Hermitian part of the spectral inputs, zero-padded inverse FFT
//            along z for every kx >= 0 (9 lines per (y, kx));
//   k_xmid : inverse FFT along x of pairs of real fields packed as one complex
//            line, the pointwise products, forward FFT along x (kx >= 0 kept);
//   k_zfwd : forward FFT along z, truncation to |k| <= K with the reference's
//            max-mode handling, and the spectral combinations the solve needs.
// The linearised equations need no transform: their terms are y-local
// multiples of spectral fields, handled by k_linear_terms.
#pragma once

#include "jsd_common.cuh"
#include "jsd_fft.cuh"

namespace jsd {

enum EqKind { kNS = 0, kPerturbation = 1, kDual = 2 };

template <typename C>
__device__ __forceinline__ void load_twiddles(C* dst, const C* __restrict__ src, int n) {
  for (int i = threadIdx.x; i < n - 1; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// inverse z pass: block (kx in [0, K], y). Inputs u, v, w and their y
// derivatives du, dv, dw (spectral). Output lines (z positions 0..pz-1) of the
// z-transformed Hermitian parts:
//   0 u, 1 v, 2 w, 3 du/dy, 4 dv/dy, 5 dw/dy, 6 du/dz, 7 dv/dz, 8 dw/dz
// stored at inter[((f * ny + y) * (K+1) + kx) * pz + z].
// ---------------------------------------------------------------------------
constexpr int kZinvLines = 9;

// Up to two sets of spectral inputs (u, v, w, du/dy, dv/dy, dw/dy): the state
// being stepped and, for the dual equations, the frozen forward state.
struct ZinvSrc {
  const double2* f[12];
  int nsets;
};

template <typename C>
__global__ void k_zinv(Geo g, FftDesc fz, const C* __restrict__ tw, ZinvSrc src, C* __restrict__ inter) {
  using Rl = typename real_of<C>::type;
  extern __shared__ __align__(16) unsigned char zsm_raw[];
  C* zsm = reinterpret_cast<C*>(zsm_raw);
  const int pz = g.pz;
  const int L = fline(pz);
  const int nl = kZinvLines * src.nsets;
  C* twl = zsm;
  C* bufa = twl + pz;
  C* bufb = bufa + nl * L;
  const int kx = blockIdx.x;
  const int y = blockIdx.y;
  load_twiddles(twl, tw, pz);
  for (int i = threadIdx.x; i < nl * L; i += blockDim.x) bufa[i] = cmake<C>(0, 0);
  __syncthreads();
  for (int i = threadIdx.x; i < 6 * src.nsets * g.mz; i += blockDim.x) {
    const int f = i / g.mz;  // input index 0 .. 6 nsets - 1
    const int iz = i - f * g.mz;
    const int set = f / 6, fi = f - set * 6;
    const int kz = signed_mode(iz, g.mz);
    const C sv = to_c<C>(sym_at(g, src.f[f], y, kx, kz));
    const int pos = fpad(kz >= 0 ? kz : pz + kz);
    C* lines = bufa + (size_t)set * kZinvLines * L;
    lines[fi * L + pos] = sv;
    if (fi < 3) lines[(6 + fi) * L + pos] = cmul_ik(sv, (Rl)(kz * g.az));
  }
  __syncthreads();
  C* res = fft_lines<true>(bufa, bufb, nl, fz, twl);
  const int K1 = g.kx_max + 1;
  for (int i = threadIdx.x; i < nl * pz; i += blockDim.x) {
    const int f = i / pz;
    const int z = i - f * pz;
    inter[(((size_t)f * g.ny + y) * K1 + kx) * pz + z] = res[f * L + fpad(z)];
  }
}

// ---------------------------------------------------------------------------
// x pass with the products: block (z block of ZB columns, y).
// Pairs of real fields are packed as a + i b into one complex line of length
// px whose spectrum is A[k] + i B[k] (k >= 0) and conj(A[k]) + i conj(B[k])
// at px - k; the inverse FFT returns a in the real and b in the imaginary part.
// Two pairs (2 ZB lines) go through each FFT batch. Every thread owns the same
// physical points in every batch (point i = threadIdx.x + e * blockDim.x), so
// the per-point fields and product accumulators stay in registers.
//
// Skew-symmetric convective term (lam = 1 for the full equations, 0 when
// linearised) plus the base-flow coupling of the perturbation equations with
// U = U(y), U' = dU/dy:
//   hel_i = -lam (u . grad) u_i + lam/2 (div u) u_i - U d_x u_i
//           - delta_i0 (v U' - (div u) U / 2)
// ---------------------------------------------------------------------------
constexpr int kXmidThreads = 256;
constexpr int kXmidEPT = 4;  // points per thread: ZB * px <= kXmidEPT * kXmidThreads

template <typename C, int ZB>
struct XmidSmem {
  static size_t bytes(const Geo& g) {
    return sizeof(C) * ((size_t)g.px + 2 * 2 * (size_t)ZB * fline(g.px));
  }
};

// Write ZB complete packed lines (zeros included) for fields (fa, fb) of the ZB
// columns starting at `line` (no barrier). Threads run x-major over (x, zl) so
// neighbouring threads read neighbouring z of one kx row of the intermediate.
template <typename C, int ZB>
__device__ __forceinline__ void fill_pair(const Geo& g, C* line, const C* __restrict__ inter, int y, int z0, int fa,
                                          bool dxa, int fb, bool dxb) {
  using Rl = typename real_of<C>::type;
  const int px = g.px, K = g.kx_max, K1 = K + 1, L = fline(px);
  for (int i = threadIdx.x; i < ZB * px; i += blockDim.x) {
    const int x = i / ZB;
    const int zl = i - x * ZB;
    const int z = z0 + zl;
    C out = cmake<C>(0, 0);
    const bool lo = x <= K, hi = x >= px - K;
    if ((lo || hi) && z < g.pz) {
      const int kx = lo ? x : px - x;
      C A = inter[(((size_t)fa * g.ny + y) * K1 + kx) * g.pz + z];
      C B = inter[(((size_t)fb * g.ny + y) * K1 + kx) * g.pz + z];
      const Rl k = (Rl)(kx * g.ax);
      if (dxa) A = cmul_ik(A, k);
      if (dxb) B = cmul_ik(B, k);
      if (x == 0) out = cmake<C>(A.x, B.x);
      else if (lo) out = cmake<C>(A.x - B.y, A.y + B.x);
      else out = cmake<C>(A.x + B.y, B.x - A.y);
    }
    line[zl * L + fpad(x)] = out;
  }
}

// fill a batch of two pairs (2 ZB lines); no barrier
template <typename C, int ZB>
__device__ __forceinline__ void fill_two_pairs(const Geo& g, C* la, const C* __restrict__ inter, int y, int z0,
                                               int fa1, bool dxa1, int fb1, bool dxb1, int fa2, bool dxa2, int fb2,
                                               bool dxb2) {
  fill_pair<C, ZB>(g, la, inter, y, z0, fa1, dxa1, fb1, dxb1);
  fill_pair<C, ZB>(g, la + ZB * fline(g.px), inter, y, z0, fa2, dxa2, fb2, dxb2);
}

// value of point i (line zl = i / px, position x) of pair set `set` in r
template <typename C>
__device__ __forceinline__ C pair_value(const C* r, int set, int zb, int px, int i) {
  const int L = fline(px);
  const int zl = i / px;
  const int x = i - zl * px;
  return r[(set * zb + zl) * L + fpad(x)];
}

// forward FFT of (h0 + i h1) and (h2 + 0 i) lines and the kx >= 0 outputs
template <typename C, int ZB>
__device__ __forceinline__ void forward_and_store(const Geo& g, const FftDesc& fx, const C* twl, C* la, C* lb,
                                                  C* __restrict__ out3, int y, int z0) {
  using Rl = typename real_of<C>::type;
  const int px = g.px, L = fline(px), K1 = g.kx_max + 1;
  C* r = fft_lines<false>(la, lb, 2 * ZB, fx, twl);
  const Rl half = (Rl)0.5;
  for (int i = threadIdx.x; i < ZB * K1; i += blockDim.x) {
    const int kx = i / ZB;
    const int zl = i - kx * ZB;
    const int z = z0 + zl;
    if (z >= g.pz) continue;
    const C a = r[zl * L + fpad(kx)];
    const C b = r[zl * L + fpad(kx == 0 ? 0 : px - kx)];
    // H0 = (Z[k] + conj Z[-k]) / 2, H1 = (Z[k] - conj Z[-k]) / (2 i)
    out3[(((size_t)0 * g.ny + y) * K1 + kx) * g.pz + z] = cmake<C>(half * (a.x + b.x), half * (a.y - b.y));
    out3[(((size_t)1 * g.ny + y) * K1 + kx) * g.pz + z] = cmake<C>(half * (a.y + b.y), -half * (a.x - b.x));
    out3[(((size_t)2 * g.ny + y) * K1 + kx) * g.pz + z] = r[(ZB + zl) * L + fpad(kx)];
  }
}

template <typename C, int ZB>
__global__ void __launch_bounds__(kXmidThreads) k_xmid(Geo g, FftDesc fx, const C* __restrict__ tw,
                                                       const C* __restrict__ inter, C* __restrict__ out3,
                                                       const double* __restrict__ ubase,
                                                       const double* __restrict__ dubase, double lam_d) {
  using Rl = typename real_of<C>::type;
  extern __shared__ __align__(16) unsigned char xsm_raw[];
  C* xsm = reinterpret_cast<C*>(xsm_raw);
  const int px = g.px, L = fline(px);
  C* twl = xsm;
  C* la = twl + px;
  C* lb = la + 2 * ZB * L;
  const int z0 = blockIdx.x * ZB;
  const int y = blockIdx.y;
  const Rl ub = ubase ? (Rl)ubase[y / g.nb] : (Rl)0;
  const Rl dub = dubase ? (Rl)dubase[y / g.nb] : (Rl)0;
  const Rl c = (Rl)g.c_inv;
  const Rl lam = (Rl)lam_d, half = (Rl)0.5;
  const int npt = ZB * px;
  load_twiddles(twl, tw, px);
  Rl U[kXmidEPT], V[kXmidEPT], W[kXmidEPT], DIV[kXmidEPT], A0[kXmidEPT], A1[kXmidEPT], A2[kXmidEPT];

  // intermediate: 0 u, 1 v, 2 w, 3 du/dy, 4 dv/dy, 5 dw/dy, 6 du/dz, 7 dv/dz, 8 dw/dz
  // Batches of two pairs; consuming batch b overlaps filling batch b + 1 when
  // the FFT result sits in lb (odd number of passes).
  fill_two_pairs<C, ZB>(g, la, inter, y, z0, 0, false, 1, false, 2, false, 0, true);
  __syncthreads();
  C* r = fft_lines<true>(la, lb, 2 * ZB, fx, twl);
#pragma unroll
  for (int e = 0; e < kXmidEPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x;
    if (i >= npt) break;
    const C p = pair_value(r, 0, ZB, px, i), q = pair_value(r, 1, ZB, px, i);
    U[e] = p.x * c;
    V[e] = p.y * c;
    W[e] = q.x * c;
    const Rl dxu = q.y * c;
    DIV[e] = dxu;
    A0[e] = lam * U[e] * dxu + ub * dxu;
  }
  if (r == la) __syncthreads();
  fill_two_pairs<C, ZB>(g, la, inter, y, z0, 4, false, 8, false, 1, true, 2, true);
  __syncthreads();
  r = fft_lines<true>(la, lb, 2 * ZB, fx, twl);
#pragma unroll
  for (int e = 0; e < kXmidEPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x;
    if (i >= npt) break;
    const C p = pair_value(r, 0, ZB, px, i), q = pair_value(r, 1, ZB, px, i);
    const Rl dyv = p.x * c, dzw = p.y * c, dxv = q.x * c, dxw = q.y * c;
    DIV[e] += dyv + dzw;
    A1[e] = lam * V[e] * dyv + lam * U[e] * dxv + ub * dxv;
    A2[e] = lam * W[e] * dzw + lam * U[e] * dxw + ub * dxw;
  }
  if (r == la) __syncthreads();
  fill_two_pairs<C, ZB>(g, la, inter, y, z0, 3, false, 5, false, 6, false, 7, false);
  __syncthreads();
  r = fft_lines<true>(la, lb, 2 * ZB, fx, twl);
#pragma unroll
  for (int e = 0; e < kXmidEPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x;
    if (i >= npt) break;
    const C p = pair_value(r, 0, ZB, px, i), q = pair_value(r, 1, ZB, px, i);
    const Rl dyu = p.x * c, dyw = p.y * c, dzu = q.x * c, dzv = q.y * c;
    A0[e] += lam * V[e] * dyu + lam * W[e] * dzu;
    A2[e] += lam * V[e] * dyw;
    A1[e] += lam * W[e] * dzv;
  }
  if (r == la) __syncthreads();
  // products packed as (hel0 + i hel1) and (hel2 + 0 i)
#pragma unroll
  for (int e = 0; e < kXmidEPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x;
    if (i >= npt) break;
    const Rl d = DIV[e];
    const Rl h0 = -A0[e] + half * lam * d * U[e] - V[e] * dub + half * d * ub;
    const Rl h1 = -A1[e] + half * lam * d * V[e];
    const Rl h2 = -A2[e] + half * lam * d * W[e];
    const int zl = i / px, x = i - zl * px;
    la[zl * L + fpad(x)] = cmake<C>(h0, h1);
    la[(ZB + zl) * L + fpad(x)] = cmake<C>(h2, (Rl)0);
  }
  __syncthreads();
  forward_and_store<C, ZB>(g, fx, twl, la, lb, out3, y, z0);
}

// ---------------------------------------------------------------------------
// x pass with the adjoint products (navier_stokes_perturbation_dual.py:214-294,
// lam = 1): dual state v, frozen forward state u, base U(y) e_x, Ut = U + u:
//   hel_i = -(Ut . grad) v_i + sum_j v_j d_i Ut_j + [(div u) v_i + (div v) Ut_i] / 4
// Intermediate lines 0..8 hold v (v, dv/dy, dv/dz), 9..17 the same for u.
// ---------------------------------------------------------------------------
template <typename C, int ZB>
__global__ void __launch_bounds__(kXmidThreads) k_xmid_dual(Geo g, FftDesc fx, const C* __restrict__ tw,
                                                            const C* __restrict__ inter, C* __restrict__ out3,
                                                            const double* __restrict__ ubase,
                                                            const double* __restrict__ dubase) {
  using Rl = typename real_of<C>::type;
  extern __shared__ __align__(16) unsigned char xsm_raw[];
  C* xsm = reinterpret_cast<C*>(xsm_raw);
  const int px = g.px, L = fline(px);
  C* twl = xsm;
  C* la = twl + px;
  C* lb = la + 2 * ZB * L;
  const int z0 = blockIdx.x * ZB;
  const int y = blockIdx.y;
  const Rl ub = (Rl)ubase[y / g.nb];
  const Rl dub = (Rl)dubase[y / g.nb];
  const Rl c = (Rl)g.c_inv;
  const Rl q4 = (Rl)0.25;
  const int npt = ZB * px;
  load_twiddles(twl, tw, px);
  Rl V0[kXmidEPT], V1[kXmidEPT], V2[kXmidEPT], U0[kXmidEPT], U1[kXmidEPT], U2[kXmidEPT];
  Rl A0[kXmidEPT], A1[kXmidEPT], A2[kXmidEPT], DV[kXmidEPT], DU[kXmidEPT];
#define JSD_EACH(body)                                                        \
  _Pragma("unroll") for (int e = 0; e < kXmidEPT; ++e) {                      \
    const int i = threadIdx.x + e * blockDim.x;                               \
    if (i >= npt) break;                                                      \
    const C p = pair_value(r, 0, ZB, px, i), q = pair_value(r, 1, ZB, px, i);  \
    const Rl pa = p.x * c, pb = p.y * c, qa = q.x * c, qb = q.y * c;          \
    body                                                                      \
  }                                                                           \
  if (r == la) __syncthreads();
#define JSD_BATCH(fa1, dxa1, fb1, dxb1, fa2, dxa2, fb2, dxb2)                   \
  fill_two_pairs<C, ZB>(g, la, inter, y, z0, fa1, dxa1, fb1, dxb1, fa2, dxa2, fb2, dxb2); \
  __syncthreads();                                                            \
  r = fft_lines<true>(la, lb, 2 * ZB, fx, twl);
  // (v0, v1) + (v2, u0)
  C* r = la;
  JSD_BATCH(0, false, 1, false, 2, false, 9, false)
  JSD_EACH(V0[e] = pa; V1[e] = pb; V2[e] = qa; U0[e] = qb;)
  // (u1, u2) + (dv0/dx, dv1/dx)
  JSD_BATCH(10, false, 11, false, 0, true, 1, true)
  JSD_EACH(U1[e] = pa; U2[e] = pb; const Rl ut = ub + U0[e]; A0[e] = -ut * qa; A1[e] = -ut * qb; DV[e] = qa;)
  // (dv2/dx, dv0/dy) + (dv1/dy, dv2/dy)
  JSD_BATCH(2, true, 3, false, 4, false, 5, false)
  JSD_EACH(A2[e] = -(ub + U0[e]) * pa; A0[e] -= U1[e] * pb; A1[e] -= U1[e] * qa; A2[e] -= U1[e] * qb;
           DV[e] += qa;)
  // (dv0/dz, dv1/dz) + (dv2/dz, du0/dx)
  JSD_BATCH(6, false, 7, false, 8, false, 9, true)
  JSD_EACH(A0[e] -= U2[e] * pa; A1[e] -= U2[e] * pb; A2[e] -= U2[e] * qa; DV[e] += qa; A0[e] += V0[e] * qb;
           DU[e] = qb;)
  // (du1/dx, du2/dx) + (du0/dy, du1/dy)
  JSD_BATCH(10, true, 11, true, 12, false, 13, false)
  JSD_EACH(A0[e] += V1[e] * pa + V2[e] * pb; A1[e] += V0[e] * qa + V1[e] * qb; DU[e] += qb;)
  // (du2/dy, du0/dz) + (du1/dz, du2/dz)
  JSD_BATCH(14, false, 15, false, 16, false, 17, false)
  JSD_EACH(A1[e] += V2[e] * pa; A2[e] += V0[e] * pb + V1[e] * qa + V2[e] * qb; DU[e] += qb;)
#undef JSD_EACH
#undef JSD_BATCH
#pragma unroll
  for (int e = 0; e < kXmidEPT; ++e) {
    const int i = threadIdx.x + e * blockDim.x;
    if (i >= npt) break;
    const Rl du = DU[e], dv = DV[e];
    const Rl h0 = A0[e] + q4 * du * V0[e] + q4 * dv * (ub + U0[e]);
    const Rl h1 = A1[e] + dub * V0[e] + q4 * du * V1[e] + q4 * dv * U1[e];
    const Rl h2 = A2[e] + q4 * du * V2[e] + q4 * dv * U2[e];
    const int zl = i / px, x = i - zl * px;
    la[zl * L + fpad(x)] = cmake<C>(h0, h1);
    la[(ZB + zl) * L + fpad(x)] = cmake<C>(h2, (Rl)0);
  }
  __syncthreads();
  forward_and_store<C, ZB>(g, fx, twl, la, lb, out3, y, z0);
}

// ---------------------------------------------------------------------------
// Outputs shared by the transform path and the linear path. For a spectral
// slot (y, ix, iz) with the three helicity components H (already truncated the
// reference's way) compute
//   q  = i kx H0 + i kz H2        (h_v = -d/dy q - k^2 H1)
//   h1 = H1
//   hg = i kz H0 - i kx H2        (h_g, navier_stokes.py:48-73)
// and record conv00 = -H at (0, 0) for the mean-flow solve.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void write_terms(const Geo& g, int y, int ix, int iz, double2 h0, double2 h1, double2 h2,
                                            double2* __restrict__ q, double2* __restrict__ H1,
                                            double2* __restrict__ hg, double2* __restrict__ conv00) {
  const double kx = kx_of(g, ix), kz = kz_of(g, iz);
  const size_t o = sidx(g, y, ix, iz);
  q[o] = cadd(cmul_ik(h0, kx), cmul_ik(h2, kz));
  H1[o] = h1;
  hg[o] = csub(cmul_ik(h0, kz), cmul_ik(h2, kx));
  if (ix == 0 && iz == 0) {
    conv00[y] = make_double2(-h0.x, -h0.y);
    conv00[g.ny + y] = make_double2(-h2.x, -h2.y);
  }
}

// Source terms of a stage (navier_stokes.py:1461-1491, 1697-1703): h_v += hv,
// h_g += hgs (spectral fields in state layout), and the (0,0) mean-flow
// forcing gains s00 = (s_x(y), s_z(y)). h_v reaches the solve only as
// -k^2 H1 (write_terms), so hv enters H1 as -hv / k^2; at kx = kz = 0 the v
// equation is not solved (the mean flow carries that mode) and the mean-flow
// forcing -conv00 + s00 takes s00 through conv00 -= s00. The source is fixed
// over the three stages of a step, so the old terms of the next stage carry it
// as the reference's do.
__global__ void k_add_source(Geo g, const double2* __restrict__ hv, const double2* __restrict__ hgs,
                             const double2* __restrict__ s00, double2* __restrict__ H1, double2* __restrict__ hg,
                             double2* __restrict__ conv00) {
  const size_t n = (size_t)g.ny * g.nk, n00 = 2 * (size_t)g.ny;
  const size_t total = n > n00 ? n : n00;
  for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < total; o += (size_t)gridDim.x * blockDim.x) {
    if (o < n) {
      const int r = (int)(o % g.nk);
      const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
      const double kx = kx_of(g, ix), kz = kz_of(g, iz);
      const double k2 = kx * kx + kz * kz;
      if (k2 > 0.0) {
        const double2 a = hv[o];
        H1[o] = make_double2(H1[o].x - a.x / k2, H1[o].y - a.y / k2);
      }
      hg[o] = cadd(hg[o], hgs[o]);
    }
    if (o < n00) conv00[o] = csub(conv00[o], s00[o]);
  }
}

// The (0, 0) column of an h_v source. There h_v = -D q - k^2 H1 reduces to
// -D q, and D has a constant null space, so the source cannot enter through q
// or H1; its interior part goes into the eigen coordinates instead:
// X1(:, (0,0)) -= V^-1 hv(interior, (0,0)). The reference adds the source to
// h_v at every wavenumber, (0, 0) included, and solves the v equation there
// as at every other wavenumber (navier_stokes.py:1697-1703). One thread per
// eigen row; single-run plans (the source is one field).
template <typename TI>
__global__ void k_add_source00(Geo g, const double* __restrict__ vinv, int lda, const double2* __restrict__ hv,
                               TI* __restrict__ X1) {
  const int n = g.ny - 2;
  const size_t N = 2 * (size_t)g.nk * g.nb;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int j = 0; j < n; ++j) {
      const double a = vinv[(size_t)i * lda + j];
      const double2 h = hv[(size_t)(j + 1) * g.nk];
      re += a * h.x;
      im += a * h.y;
    }
    X1[(size_t)i * N] = (TI)((double)X1[(size_t)i * N] - re);
    X1[(size_t)i * N + 1] = (TI)((double)X1[(size_t)i * N + 1] - im);
  }
}

// forward z pass: block (kx in [0, K], y).
template <typename C>
__global__ void k_zfwd(Geo g, FftDesc fz, const C* __restrict__ tw, const C* __restrict__ out3,
                       double2* __restrict__ q, double2* __restrict__ H1, double2* __restrict__ hg,
                       double2* __restrict__ conv00) {
  extern __shared__ __align__(16) unsigned char fsm_raw[];
  C* fsm = reinterpret_cast<C*>(fsm_raw);
  const int pz = g.pz;
  const int L = fline(pz);
  C* twl = fsm;
  C* bufa = twl + pz;
  C* bufb = bufa + 3 * L;
  const int kx = blockIdx.x;
  const int y = blockIdx.y;
  const int K1 = g.kx_max + 1;
  load_twiddles(twl, tw, pz);
  for (int i = threadIdx.x; i < 3 * pz; i += blockDim.x) {
    const int f = i / pz;
    const int z = i - f * pz;
    bufa[f * L + fpad(z)] = out3[(((size_t)f * g.ny + y) * K1 + kx) * pz + z];
  }
  __syncthreads();
  C* F = fft_lines<false>(bufa, bufb, 3, fz, twl);
  const double cf = g.c_fwd;
  auto getF = [&](int f, int kz) -> double2 {
    const C v = F[f * L + fpad(kz >= 0 ? kz : pz + kz)];
    return make_double2((double)v.x * cf, (double)v.y * cf);
  };
  const int K = g.kx_max;
  // rows this block owns: kx itself; -kx for 1 <= kx < K; the -K slot when kx = K
  int rows[2];
  int nrows = 1;
  rows[0] = kx;
  if (kx >= 1 && kx < K) rows[nrows++] = g.mx - kx;
  if (kx == K) rows[nrows++] = K + 1;
  for (int i = threadIdx.x; i < nrows * g.mz; i += blockDim.x) {
    const int rr = i / g.mz;
    const int iz = i - rr * g.mz;
    const int ix = rows[rr];
    int sx, sz;
    bool cj;
    truncation_source(g, ix, iz, sx, sz, cj);
    // true coefficient at (sx, sz): sx >= 0 here except for rows -kx
    double2 h[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      double2 val = (sx >= 0) ? getF(f, sz) : cconj(getF(f, -sz));
      h[f] = cj ? cconj(val) : val;
    }
    write_terms(g, y, ix, iz, h[0], h[1], h[2], q, H1, hg, conv00);
  }
}

// ---------------------------------------------------------------------------
// Linearised equations: every term is a y-dependent multiple of a spectral
// field, so hat(no_hat(.) * U(y)) = U(y) * RT(.), where RT is the round trip
// "Hermitian part, then the reference truncation". Thread per output slot.
//   perturbation (navier_stokes_perturbation.py:160-239, lam = 0):
//     P0 = -U i kx u - U' v + U div(u) / 2,  P1 = -U i kx v,  P2 = -U i kx w
//   dual (navier_stokes_perturbation_dual.py:214-294, lam = 0, base (U, 0, 0)):
//     P0 = -U i kx u + U div(u) / 4,  P1 = -U i kx v + U' u,  P2 = -U i kx w
// ---------------------------------------------------------------------------
template <int KIND>
__device__ __forceinline__ void linear_pre(const Geo& g, const double2* __restrict__ u, const double2* __restrict__ v,
                                           const double2* __restrict__ w, const double2* __restrict__ dv, int y,
                                           int kx, int kz, double ub, double dub, double2* P) {
  const size_t o = sidx(g, y, mode_pos(kx, g.mx), mode_pos(kz, g.mz));
  const double2 uu = u[o], vv = v[o], ww = w[o], dvv = dv[o];
  const double kxv = kx * g.ax, kzv = kz * g.az;
  const double2 div = cadd(cadd(cmul_ik(uu, kxv), dvv), cmul_ik(ww, kzv));
  if (KIND == kPerturbation) {
    P[0] = cadd(csub(cscale(cmul_ik(uu, kxv), -ub), cscale(vv, dub)), cscale(div, 0.5 * ub));
    P[1] = cscale(cmul_ik(vv, kxv), -ub);
  } else {
    P[0] = cadd(cscale(cmul_ik(uu, kxv), -ub), cscale(div, 0.25 * ub));
    P[1] = cadd(cscale(cmul_ik(vv, kxv), -ub), cscale(uu, dub));
  }
  P[2] = cscale(cmul_ik(ww, kxv), -ub);
}

template <int KIND>
__global__ void k_linear_terms(Geo g, const double2* __restrict__ u, const double2* __restrict__ v,
                               const double2* __restrict__ w, const double2* __restrict__ dv,
                               const double* __restrict__ ubase, const double* __restrict__ dubase,
                               double2* __restrict__ q, double2* __restrict__ H1, double2* __restrict__ hg,
                               double2* __restrict__ conv00) {
  const size_t total = (size_t)g.ny * g.nk;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(t / g.nk);
    const int r = (int)(t - (size_t)y * g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    int sx, sz;
    bool cj;
    truncation_source(g, ix, iz, sx, sz, cj);
    const double ub = ubase[y / g.nb], dub = dubase[y / g.nb];
    double2 Pa[3], Pb[3];
    linear_pre<KIND>(g, u, v, w, dv, y, sx, sz, ub, dub, Pa);
    linear_pre<KIND>(g, u, v, w, dv, y, -sx, -sz, ub, dub, Pb);
    double2 h[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const double2 s = make_double2(0.5 * (Pa[f].x + Pb[f].x), 0.5 * (Pa[f].y - Pb[f].y));
      h[f] = cj ? cconj(s) : s;
    }
    write_terms(g, y, ix, iz, h[0], h[1], h[2], q, H1, hg, conv00);
  }
}

// coupling_term = False (navier_stokes_perturbation.py:217-237,
// navier_stokes_perturbation_dual.py:270-292): with C = hat(U'(y) f) =
// U'(y) RT(f) (RT = Hermitian part, then the reference truncation)
//   perturbation: h_g += i kz C  with f = v (wall-normal velocity);
//   dual:         h_v += d_x^2 C + d_z^2 C = -k^2 C, i.e. H1 += C, with f = the
//                 streamwise component of the dual field.
// g.ny = planes (batch runs included); dubase indexed by Chebyshev row.
template <int KIND>
__global__ void k_coupling_off(Geo g, const double2* __restrict__ f, const double* __restrict__ dubase,
                               double2* __restrict__ H1, double2* __restrict__ hg) {
  const size_t total = (size_t)g.ny * g.nk;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(t / g.nk);
    const int r = (int)(t - (size_t)y * g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    int sx, sz;
    bool cj;
    truncation_source(g, ix, iz, sx, sz, cj);
    double2 c = sym_at(g, f, y, sx, sz);
    if (cj) c = cconj(c);
    c = cscale(c, dubase[y / g.nb]);
    if (KIND == kPerturbation) {
      hg[t] = cadd(hg[t], cmul_ik(c, kz_of(g, iz)));
    } else {
      H1[t] = cadd(H1[t], c);
    }
  }
}

// omega_y = i kz u - i kx w (the y component of curl u, domain.py:920-933)
__global__ void k_omega(Geo g, const double2* __restrict__ u, const double2* __restrict__ w,
                        double2* __restrict__ om) {
  const size_t total = (size_t)g.ny * g.nk;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(t % g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    om[t] = csub(cmul_ik(u[t], kz_of(g, iz)), cmul_ik(w[t], kx_of(g, ix)));
  }
}

// ---------------------------------------------------------------------------
// Per-column eigenbasis update of the Helmholtz / Poisson / influence-matrix
// solve (navier_stokes.py:1291-1414). In the eigenbasis D2_int = V diag(lam) V^-1
// every per-wavenumber operator is diagonal; L_j = lam_j - k^2:
//   h_v~   = -X1 - k^2 H1~                        (h_v = -D q - k^2 H1)
//   phi~   = L v~ + c0 v(+1) + cN v(-1)           (phi = lap v, interior)
//   v_p~   = (R phi~ + dt_e (gamma h_v~ + xi h_v,old~)) / (H L)
//   v_a~   = (beta dt / Re) c0 / (H L),  v_b~ = sgn v_a~   (v_b = flip v_a)
//   [a b]  = M^-1 [-(w0 . v_p~), -(wN . v_p~)]  with M from w0, wN . v_a~, v_b~
//   v~     = v_p~ + (a + b sgn) v_a~
//   om~    = (R om~ + dt_e (gamma h_g~ + xi h_g,old~)) / H
// with R = 1 + alpha dt/Re L, H = 1 - beta dt/Re L. One thread per real column.
// ---------------------------------------------------------------------------
struct EigTables {
  const double* lam;
  const double* c0;
  const double* cN;
  const double* sgn;
  const double* w0;
  const double* wN;
  const double* re_run;  // Reynolds number per run of a batch (nullptr: StageCoef::re)
};

struct StageCoef {
  double alpha, beta, gamma, xi;
  double dt, dt_e, re;
  int first;  // the previous-stage terms are zero
};

constexpr int kEigCols = 32;    // columns per block (one warp-wide row segment)
constexpr int kEigParts = 4;    // warps per block, each walking a quarter of the eigen rows
constexpr int kEigBatch = 4;    // rows whose loads are issued together (loads in flight per thread: 7 x batch)

// Rows of a block's part: j1 - j0 <= ceil((Ny - 2) / kEigParts). The first
// pass keeps v_p~ of its rows in shared memory for the second (rpp rows per
// part, dynamic shared memory of eigen_update_smem bytes).
inline int eigen_update_rpp(int ny) { return (ny - 2 + kEigParts - 1) / kEigParts; }
inline size_t eigen_update_smem(int ny) { return sizeof(double) * kEigParts * eigen_update_rpp(ny) * kEigCols; }

// TI: storage of the nonlinear terms (X1, H1~, h_g~ and the previous stage's
// h_v~, h_g~): double, or float where they come out of FP32 transforms and
// products (the mixed form)
template <typename TI>
__global__ void __launch_bounds__(kEigCols * kEigParts, 4) k_eigen_update(
    Geo g, EigTables t, StageCoef sc, const TI* __restrict__ X1, const TI* __restrict__ H1t,
    const TI* __restrict__ hgt, const double* __restrict__ vt, const double* __restrict__ omt,
    const double* __restrict__ vfield, TI* __restrict__ hv_old, TI* __restrict__ hg_old,
    double* __restrict__ vnt, double* __restrict__ omnt, int rpp) {
  __shared__ double red[kEigParts][6][kEigCols];
  extern __shared__ double vps_all[];
  const int N = 2 * g.nk * g.nb;  // columns: real and imaginary parts of every mode of every run
  const int lane = threadIdx.x % kEigCols;
  const int part = threadIdx.x / kEigCols;
  const int c = blockIdx.x * kEigCols + lane;
  const bool active = c < N;
  const int n = g.ny - 2;
  const int j0 = (n * part) / kEigParts, j1 = (n * (part + 1)) / kEigParts;
  double* vps = vps_all + (size_t)part * rpp * kEigCols + lane;  // v_p~ of row j at vps[(j - j0) * kEigCols]
  double k2 = 0.0, v0 = 0.0, vN = 0.0, re = sc.re;
  if (active) {
    const int run = (c >> 1) / g.nk;
    const int kp = (c >> 1) - run * g.nk;
    const int ix = kp / g.mz, iz = kp - (kp / g.mz) * g.mz;
    const double kx = kx_of(g, ix), kz = kz_of(g, iz);
    k2 = kx * kx + kz * kz;
    v0 = vfield[c];
    vN = vfield[(size_t)(g.ny - 1) * N + c];
    if (t.re_run) re = t.re_run[run];
  }
  const double ar = sc.alpha * sc.dt / re;
  const double br = sc.beta * sc.dt / re;
  double d0p = 0, dNp = 0, d0a = 0, dNa = 0, d0b = 0, dNb = 0;
  if (active) {
    // rows whose loads are in flight together: more when the terms are FP32
    constexpr int NB = sizeof(TI) == 4 ? 2 * kEigBatch : kEigBatch;
    for (int jb = j0; jb < j1; jb += NB) {
      // all loads of the batch first (independent rows), then the arithmetic
      TI x1[NB], h1[NB], hg[NB], hvo[NB], hgo[NB];
      double vv[NB], om[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int j = jb + b;
        x1[b] = h1[b] = hg[b] = hvo[b] = hgo[b] = (TI)0;
        vv[b] = om[b] = 0.0;
        if (j < j1) {
          const size_t o = (size_t)j * N + c;
          x1[b] = X1[o];
          h1[b] = H1t[o];
          hg[b] = hgt[o];
          vv[b] = vt[o];
          om[b] = omt[o];
          if (!sc.first) {
            hvo[b] = hv_old[o];
            hgo[b] = hg_old[o];
          }
        }
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const int j = jb + b;
        if (j >= j1) break;
        const size_t o = (size_t)j * N + c;
        const double L = t.lam[j] - k2;
        const double R = 1.0 + ar * L;
        const double H = 1.0 - br * L;
        const double ihl = 1.0 / (H * L);  // one reciprocal: 1 / H = L / (H L)
        const double ih = L * ihl;
        const double hv = -(double)x1[b] - k2 * (double)h1[b];
        const double phi = L * vv[b] + t.c0[j] * v0 + t.cN[j] * vN;
        const double vp = (R * phi + sc.dt_e * (sc.gamma * hv + sc.xi * (double)hvo[b])) * ihl;
        const double va = br * t.c0[j] * ihl;
        const double w0 = t.w0[j], wN = t.wN[j], sg = t.sgn[j];
        d0p += w0 * vp;
        dNp += wN * vp;
        d0a += w0 * va;
        dNa += wN * va;
        d0b += w0 * sg * va;
        dNb += wN * sg * va;
        vps[(j - j0) * kEigCols] = vp;
        hv_old[o] = (TI)hv;
        omnt[o] = (R * om[b] + sc.dt_e * (sc.gamma * (double)hg[b] + sc.xi * (double)hgo[b])) * ih;
        hg_old[o] = hg[b];
      }
    }
  }
  red[part][0][lane] = d0p;
  red[part][1][lane] = dNp;
  red[part][2][lane] = d0a;
  red[part][3][lane] = dNa;
  red[part][4][lane] = d0b;
  red[part][5][lane] = dNb;
  __syncthreads();
  if (!active) return;
  double sum[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double acc = 0.0;
#pragma unroll
    for (int pp = 0; pp < kEigParts; ++pp) acc += red[pp][q][lane];
    sum[q] = acc;
  }
  const double det = sum[2] * sum[5] - sum[4] * sum[3];
  const double ra = -sum[0], rb = -sum[1];
  const double a = (sum[5] * ra - sum[4] * rb) / det;
  const double b = (-sum[3] * ra + sum[2] * rb) / det;
  for (int j = j0; j < j1; ++j) {
    const double L = t.lam[j] - k2;
    const double H = 1.0 - br * L;
    const double va = br * t.c0[j] * (1.0 / (H * L));
    vnt[(size_t)j * N + c] = vps[(j - j0) * kEigCols] + (a + b * t.sgn[j]) * va;
  }
}

// ---------------------------------------------------------------------------
// (0,0) mean flow: the reference's 2Ny x 2Ny system for (U00, W00)
// (navier_stokes.py:1417-1504) with its own matrices:
//   x_new = Linv_ns (R_ns x + dt_e gamma N + dt_e xi N_old),
//   N = [-conv00_x - dpdx * scale, -conv00_z]
// One block per run (g.ny = Chebyshev points, g.nb runs; conv entries per plane,
// matrices and uw00 per run). conv_old == nullptr means zero.
// ---------------------------------------------------------------------------
constexpr int kMeanFlowThreads = 1024;

__global__ void __launch_bounds__(kMeanFlowThreads) k_mean_flow(
    Geo g, const double* __restrict__ rhs_ns, const double* __restrict__ lhs_inv_ns, const double2* __restrict__ u,
    const double2* __restrict__ w, const double2* __restrict__ conv, const double2* __restrict__ conv_old,
    const double* __restrict__ dpdx, double dpdx_scale, double dt_gamma, double dt_xi, double2* __restrict__ uw00) {
  extern __shared__ __align__(16) double2 msm[];
  const int n = g.ny, n2 = 2 * g.ny;
  // block = run of a batch: its matrices, its planes (y * nb + run) and conv entries
  const int run = blockIdx.x, nb = g.nb;
  rhs_ns += (size_t)run * 3 * n2 * n2;
  lhs_inv_ns += (size_t)run * 3 * n2 * n2;
  uw00 += (size_t)run * n2;
  double2* xv = msm;       // current (U00, W00)
  double2* rv = xv + n2;   // right-hand side
  const double dp = dpdx ? dpdx[0] * dpdx_scale : 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  auto cidx = [&](int i) { return (i < n) ? i * nb + run : n * nb + (i - n) * nb + run; };
  for (int i = threadIdx.x; i < n2; i += blockDim.x) {
    xv[i] = (i < n) ? u[sidx(g, i * nb + run, 0, 0)] : w[sidx(g, (i - n) * nb + run, 0, 0)];
  }
  __syncthreads();
  // one warp per row, lanes along the row (coalesced)
  for (int i = warp; i < n2; i += nwarps) {
    const double* row = rhs_ns + (size_t)i * n2;
    double ax = 0.0, ay = 0.0;
    for (int j = lane; j < n2; j += 32) {
      ax += xv[j].x * row[j];
      ay += xv[j].y * row[j];
    }
    for (int o = 16; o > 0; o >>= 1) {
      ax += __shfl_down_sync(0xffffffffu, ax, o);
      ay += __shfl_down_sync(0xffffffffu, ay, o);
    }
    if (lane == 0) {
      const double src = (i < n) ? -dp : 0.0;
      const double2 nn = make_double2(-conv[cidx(i)].x + src, -conv[cidx(i)].y);
      const double2 no =
          conv_old ? make_double2(-conv_old[cidx(i)].x + src, -conv_old[cidx(i)].y) : make_double2(src, 0.0);
      rv[i] = cadd(cadd(make_double2(ax, ay), cscale(nn, dt_gamma)), cscale(no, dt_xi));
    }
  }
  __syncthreads();
  for (int i = warp; i < n2; i += nwarps) {
    const double* row = lhs_inv_ns + (size_t)i * n2;
    double ax = 0.0, ay = 0.0;
    for (int j = lane; j < n2; j += 32) {
      ax += rv[j].x * row[j];
      ay += rv[j].y * row[j];
    }
    for (int o = 16; o > 0; o >>= 1) {
      ax += __shfl_down_sync(0xffffffffu, ax, o);
      ay += __shfl_down_sync(0xffffffffu, ay, o);
    }
    if (lane == 0) uw00[i] = make_double2(ax, ay);
  }
}

// Row-parallel form of the same update with LR = Linv_ns R_ns precomputed per
// stage: x_new = LR x + Linv_ns (dt_e gamma N + dt_e xi N_old). Grid (row
// blocks, runs), one warp per output row; every block first builds x and the
// forcing f = dt_e gamma N + dt_e xi N_old of its run in shared memory.
constexpr int kMeanFlowRows = 8;  // rows (warps) per block

__global__ void __launch_bounds__(32 * kMeanFlowRows) k_mean_flow_rows(
    Geo g, const double* __restrict__ lr_ns, const double* __restrict__ lhs_inv_ns, const double2* __restrict__ u,
    const double2* __restrict__ w, const double2* __restrict__ conv, const double2* __restrict__ conv_old,
    const double* __restrict__ dpdx, double dpdx_scale, double dt_gamma, double dt_xi, double2* __restrict__ uw00) {
  extern __shared__ __align__(16) double2 msm[];
  const int n = g.ny, n2 = 2 * g.ny;
  const int run = blockIdx.y, nb = g.nb;
  lr_ns += (size_t)run * 3 * n2 * n2;
  lhs_inv_ns += (size_t)run * 3 * n2 * n2;
  uw00 += (size_t)run * n2;
  double2* xv = msm;      // (U00, W00) of the run
  double2* fv = xv + n2;  // forcing
  const double dp = dpdx ? dpdx[0] * dpdx_scale : 0.0;
  for (int i = threadIdx.x; i < n2; i += blockDim.x) {
    const int ci = (i < n) ? i * nb + run : n * nb + (i - n) * nb + run;
    xv[i] = (i < n) ? u[sidx(g, i * nb + run, 0, 0)] : w[sidx(g, (i - n) * nb + run, 0, 0)];
    const double src = (i < n) ? -dp : 0.0;
    const double2 nn = make_double2(-conv[ci].x + src, -conv[ci].y);
    const double2 no = conv_old ? make_double2(-conv_old[ci].x + src, -conv_old[ci].y) : make_double2(src, 0.0);
    fv[i] = cadd(cscale(nn, dt_gamma), cscale(no, dt_xi));
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kMeanFlowRows + (threadIdx.x >> 5);
  if (i >= n2) return;
  const double* lr = lr_ns + (size_t)i * n2;
  const double* li = lhs_inv_ns + (size_t)i * n2;
  double ax = 0.0, ay = 0.0;
  for (int j = lane; j < n2; j += 32) {
    ax += lr[j] * xv[j].x + li[j] * fv[j].x;
    ay += lr[j] * xv[j].y + li[j] * fv[j].y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
  }
  if (lane == 0) uw00[i] = make_double2(ax, ay);
}

// u, w from continuity and omega_y (rk_not_00, navier_stokes.py:1506-1527);
// the (0,0) mode from the mean-flow solve; walls zeroed (domain.py:630-647).
// (g.ny = Chebyshev points, g.nb runs; uw00 holds 2 Ny entries per run)
// u, w of the new state from continuity, the (0,0) mean flow and the wall
// rows; raises kErrNonFinite in `err` when any value it reads (dv/dy, omega_y
// and the mean flow, from which all of u, v, w follow) is not finite.
__global__ void k_reconstruct(Geo g, const double2* __restrict__ dvn, const double2* __restrict__ omn,
                              const double2* __restrict__ uw00, double2* __restrict__ u, double2* __restrict__ v,
                              double2* __restrict__ w, int* __restrict__ err) {
  const size_t total = (size_t)g.ny * g.nb * g.nk;
  bool bad = false;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int plane = (int)(t / g.nk);
    const int r = (int)(t - (size_t)plane * g.nk);
    const int y = plane / g.nb, run = plane - y * g.nb;
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    if (y == 0 || y == g.ny - 1) {
      u[t] = v[t] = w[t] = make_double2(0.0, 0.0);
      continue;
    }
    if (ix == 0 && iz == 0) {
      const double2 a = uw00[(size_t)run * 2 * g.ny + y], c = uw00[(size_t)run * 2 * g.ny + g.ny + y];
      bad |= !(isfinite(a.x) && isfinite(a.y) && isfinite(c.x) && isfinite(c.y));
      u[t] = a;
      w[t] = c;
      continue;
    }
    const double kx = kx_of(g, ix), kz = kz_of(g, iz);
    const double mk2 = -(kx * kx + kz * kz);
    const double2 dv = dvn[t], om = omn[t];
    bad |= !(isfinite(dv.x) && isfinite(dv.y) && isfinite(om.x) && isfinite(om.y));
    const double2 uu = cadd(cmul_ik(dv, -kx), cmul_ik(om, kz));
    const double2 ww = csub(cmul_ik(dv, -kz), cmul_ik(om, kx));
    u[t] = make_double2(uu.x / mk2, uu.y / mk2);
    w[t] = make_double2(ww.x / mk2, ww.y / mk2);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, kErrNonFinite);
}

// ---------------------------------------------------------------------------
// Reductions. Both use a fixed order (per-plane partial sums, then one block
// sums the planes) so results are reproducible run to run.
// plane_sums: per y, sum over all modes of |Sym(f)|^2 over the three
// components (mode = 0) or of Re f (mode = 1, one component).
// ---------------------------------------------------------------------------
__global__ void k_plane_sums(Geo g, const double2* __restrict__ f, int ncomp, int mode, double* __restrict__ out) {
  const int y = blockIdx.x;
  double acc = 0.0;
  const size_t fs = (size_t)g.ny * g.nk;
  for (int r = threadIdx.x; r < g.nk; r += blockDim.x) {
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    if (mode == 0) {
      for (int c = 0; c < ncomp; ++c) {
        const double2 s = sym_at(g, f + c * fs, y, signed_mode(ix, g.mx), signed_mode(iz, g.mz));
        acc += s.x * s.x + s.y * s.y;
      }
    } else {
      acc += f[sidx(g, y, ix, iz)].x;
    }
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double a = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) out[y] = a;
  }
}

// out[0] = scale * sum_y weights[y] * partial[y]
__global__ void k_weighted_total(int ny, const double* __restrict__ weights, const double* __restrict__ partial,
                                 double scale, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double acc = 0.0;
    for (int y = 0; y < ny; ++y) acc += weights[y] * partial[y];
    out[0] = scale * acc;
  }
}

// Sliced form for the plan's reductions: block (plane, slice) sums one of
// kSumSlices contiguous slices of the plane's modes; out[plane * kSumSlices +
// slice]. Same terms as k_plane_sums, summed in a fixed order.
constexpr int kSumSlices = 8;

__global__ void __launch_bounds__(256) k_plane_sums_sliced(Geo g, const double2* __restrict__ f, int ncomp, int mode,
                                                          double* __restrict__ out) {
  const int y = blockIdx.x, slice = blockIdx.y;
  const int chunk = (g.nk + kSumSlices - 1) / kSumSlices;
  const int r0 = slice * chunk, r1 = min(g.nk, r0 + chunk);
  const size_t fs = (size_t)g.ny * g.nk;
  double acc = 0.0;
  if (mode == 0) {
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
      for (int c = 0; c < ncomp; ++c) {
        const double2 sv = sym_at(g, f + c * fs, y, signed_mode(ix, g.mx), signed_mode(iz, g.mz));
        acc += sv.x * sv.x + sv.y * sv.y;
      }
    }
  } else {
    const double2* row = f + (size_t)y * g.nk;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) acc += row[r].x;
  }
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double a = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) out[(size_t)y * kSumSlices + slice] = a;
  }
}

// One warp: sum_y w_y sum_s partial[(y * stride + offset) * kSumSlices + s], fixed order
__device__ __forceinline__ double weighted_slices(int ny, int stride, int offset, const double* __restrict__ weights,
                                                  const double* __restrict__ partial) {
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int y = lane; y < ny; y += 32) {
    const double* p = partial + ((size_t)y * stride + offset) * kSumSlices;
    double sy = 0.0;
#pragma unroll
    for (int sl = 0; sl < kSumSlices; ++sl) sy += p[sl];
    acc += weights[y] * sy;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  return acc;  // valid in lane 0
}

// out = scale * sum over planes (single run), one warp
__global__ void k_weighted_total_sliced(int ny, const double* __restrict__ weights,
                                        const double* __restrict__ partial, double scale, double* __restrict__ out) {
  const double a = weighted_slices(ny, 1, 0, weights, partial);
  if (threadIdx.x == 0) out[0] = scale * a;
}

// per-run totals of a batch: one warp per run
__global__ void k_weighted_total_runs_sliced(int ny, int nb, const double* __restrict__ weights,
                                             const double* __restrict__ partial, double scale,
                                             double* __restrict__ out) {
  const int run = blockIdx.x;
  const double a = weighted_slices(ny, nb, run, weights, partial);
  if (threadIdx.x == 0) out[run] = scale * a;
}

// mass-flux scalar from sliced partial sums of Re u, one warp
__global__ void k_mass_flux_scalar_sliced(int ny, const double* __restrict__ weights,
                                          const double* __restrict__ partial, double c_inv, double q0, double dt_e,
                                          double* __restrict__ dpdx, double* __restrict__ qdiff) {
  const double a = weighted_slices(ny, 1, 0, weights, partial);
  if (threadIdx.x == 0) {
    const double d = c_inv * a - q0;
    dpdx[0] = dpdx[0] + d / dt_e;
    qdiff[0] = d;
  }
}

// Per-run totals of a batch: out[run] = scale * sum_y w_y partial[y * nb + run]
// (partial per plane from k_plane_sums).
__global__ void k_weighted_total_runs(int ny, int nb, const double* __restrict__ weights,
                                      const double* __restrict__ partial, double scale, double* __restrict__ out) {
  const int run = blockIdx.x * blockDim.x + threadIdx.x;
  if (run >= nb) return;
  double acc = 0.0;
  for (int y = 0; y < ny; ++y) acc += weights[y] * partial[(size_t)y * nb + run];
  out[run] = scale * acc;
}

// Constant mass flux (navier_stokes.py:724-805, 1205-1214): with the flow rate
// Q = c_inv * sum_y w_y sum_k Re u(y, k) (the y-integral of u at x = z = 0),
//   dPdx += (Q - Q0) / dt_e,   u <- RT(u) + const
// where the constant is -(Q - Q0) / 2 in physical units (walls included).
__global__ void k_mass_flux_scalar(int ny, const double* __restrict__ weights, const double* __restrict__ partial,
                                   double c_inv, double q0, double dt_e, double* __restrict__ dpdx,
                                   double* __restrict__ qdiff) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double acc = 0.0;
    for (int y = 0; y < ny; ++y) acc += weights[y] * partial[y];
    const double q = c_inv * acc;
    const double d = q - q0;
    dpdx[0] = dpdx[0] + d / dt_e;
    qdiff[0] = d;
  }
}

__global__ void k_roundtrip_shift(Geo g, const double2* __restrict__ f, const double* __restrict__ qdiff,
                                  double2* __restrict__ out) {
  const size_t total = (size_t)g.ny * g.nk;
  const double shift = -qdiff[0] * 0.5 / g.c_inv;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(t / g.nk);
    const int r = (int)(t - (size_t)y * g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    int sx, sz;
    bool cj;
    truncation_source(g, ix, iz, sx, sz, cj);
    double2 s = sym_at(g, f, y, sx, sz);
    if (cj) s = cconj(s);
    if (ix == 0 && iz == 0) s.x += shift;
    out[t] = s;
  }
}

}  // namespace jsd
