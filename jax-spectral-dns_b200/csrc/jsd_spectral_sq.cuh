// Transform kernels of the nonlinear terms on register-resident square FFTs
// (jsd_fftsq.cuh), used when the plan's FFT lengths are S * S. Same three
// passes and the same intermediate layouts as the shared-memory kernels in
// jsd_spectral.cuh, with one line per group of S lanes:
//   k_zinv_sq : group per (y, kx): Hermitian part, 9 (18) inverse z transforms;
//   k_xmid_sq : block per (y, run of z columns), group per z column: packed
//               pairs of fields through inverse x transforms, the products in
//               registers (every lane owns the same x positions in every line),
//               2 forward x transforms;
//   k_zfwd_sq : group per (y, kx): 3 forward z transforms, truncation and the
//               spectral combinations of write_terms.
// All sizes are compile-time, so index arithmetic is shifts and multiplies,
// and the only synchronisation inside a transform is a __syncwarp.
#pragma once

#include "jsd_fftsq.cuh"
#include "jsd_gemm.cuh"
#include "jsd_spectral.cuh"

namespace jsd {

constexpr int kSqWarps = 4;  // warps per block

// Lane roles. HW: with two groups per warp (11 <= S <= 16) each group takes
// its own half-warp (lanes 16 gi + t, t < S): a 64-bit shared-memory request
// is served per half-warp, so the groups' accesses never share a bank cycle.
// Otherwise 32 / S groups of S consecutive lanes, the last 32 - G S idle.
template <int S, bool HW = true>
struct SqLane {
  static constexpr int G = 32 / S;                        // line groups per warp
  static constexpr int W = (HW && G == 2) ? 16 : S;       // lane stride of the groups
  int warp, gi, t;
  bool live;  // lane belongs to a group (the other lanes idle)
  __device__ __forceinline__ SqLane() {
    const int lane = threadIdx.x & 31;
    warp = threadIdx.x >> 5;
    gi = lane / W;
    t = lane - gi * W;
    live = gi < G && t < S;
    if (!live) {
      gi = 0;
      if (HW) t = 0;
    }
  }
};

// src.f[i] by selects over the parameter array (a runtime index into the
// kernel parameter would copy the array to local memory)
__device__ __forceinline__ const double2* zinv_field(const ZinvSrc& src, int i) {
  const double2* r = src.f[0];
#pragma unroll
  for (int k = 1; k < 12; ++k)
    if (i == k) r = src.f[k];
  return r;
}

// ---------------------------------------------------------------------------
// inverse z pass (same output as k_zinv)
// ---------------------------------------------------------------------------
template <typename C, int S>
__global__ void __launch_bounds__(kSqWarps * 32) k_zinv_sq(Geo g, const C* __restrict__ twtab, ZinvSrc src,
                                                           C* __restrict__ inter) {
  using Rl = typename real_of<C>::type;
  constexpr int N = S * S, XB = sq_xbuf<S>();
  // The two forms keep their best measured shapes: FP32 lines on half-warp
  // groups with the next field's rows prefetched into L2 and per-position
  // bound tests resolved at compile time; FP64 lines on consecutive-lane
  // groups with plain bound tests and no prefetch (the compiler then keeps
  // all 2 S loads of a line in flight; with the FP32 shape the FP64 pass
  // took 175 us instead of 109 us cold at 128 x 129 x 128).
  constexpr bool F32 = sizeof(C) == sizeof(float2);
  extern __shared__ __align__(16) unsigned char sq_raw[];
  const SqLane<S, F32> ln;
  C* xb = reinterpret_cast<C*>(sq_raw) + (ln.warp * SqLane<S>::G + ln.gi) * XB;
  const int K1 = g.kx_max + 1, K = g.kz_max;
  const int pair = (blockIdx.x * kSqWarps + ln.warp) * SqLane<S>::G + ln.gi;
  const bool act = ln.live && pair < g.ny * K1;
  const int y = act ? pair / K1 : 0;
  const int kx = act ? pair - y * K1 : 0;
  C tw[S - 1];
  sq_twiddles<S>(tw, twtab, ln.t);
  // the group's two rows (kx and -kx) of field `i` into L2: the loads of a
  // field then wait for L2, not DRAM (one field ahead; rows are 16-byte
  // aligned and mz * 16 bytes long)
  auto prefetch = [&](int i) {
    if (F32 && act && ln.t == 0 && i < 6 * src.nsets) {
      const double2* f = zinv_field(src, i);
      l2_prefetch(f + sidx(g, y, kx, 0), (unsigned)(g.mz * sizeof(double2)));
      if (kx) l2_prefetch(f + sidx(g, y, g.mx - kx, 0), (unsigned)(g.mz * sizeof(double2)));
    }
  };
  prefetch(1);
#pragma unroll 1
  for (int set = 0; set < src.nsets; ++set) {
#pragma unroll 1
    for (int fi = 0; fi < 6; ++fi) {
      const double2* f = zinv_field(src, set * 6 + fi);
      prefetch(set * 6 + fi + 2);
      C x[S], xz[S];
      // K < N / 2: positions below N / 2 hold kz >= 0 modes, those above kz < 0
#pragma unroll
      for (int m = 0; m < S; ++m) {
        const int p = ln.t + S * m;
        const bool below = F32 && S * m + S - 1 < N / 2, above = F32 && S * m >= N / 2;
        const bool lo = !above && p <= K, hi = !below && p >= N - K;
        const int kz = below ? p : above ? p - N : lo ? p : p - N;
        const C v = (act && (lo || hi)) ? to_c<C>(sym_at(g, f, y, kx, kz)) : cmake<C>(0, 0);
        x[m] = v;
        xz[m] = cmul_ik(v, (Rl)(kz * g.az));
      }
      sq_fft<S, true>(x, tw, xb, ln.t, ln.live);
      C* o = inter + (((size_t)(set * kZinvLines + fi) * g.ny + y) * K1 + kx) * N + ln.t;
      if (act) {
#pragma unroll
        for (int m = 0; m < S; ++m) o[S * m] = x[m];
      }
      if (fi < 3) {
        sq_fft<S, true>(xz, tw, xb, ln.t, ln.live);
        C* oz = inter + (((size_t)(set * kZinvLines + 6 + fi) * g.ny + y) * K1 + kx) * N + ln.t;
        if (act) {
#pragma unroll
          for (int m = 0; m < S; ++m) oz[S * m] = xz[m];
        }
      }
    }
  }
}

template <typename C, int S>
size_t zinv_sq_smem() {
  return sizeof(C) * (size_t)kSqWarps * SqLane<S>::G * sq_xbuf<S>();
}

// ---------------------------------------------------------------------------
// forward z pass (same output as k_zfwd)
// ---------------------------------------------------------------------------
template <typename C, int S>
__global__ void __launch_bounds__(kSqWarps * 32) k_zfwd_sq(Geo g, const C* __restrict__ twtab,
                                                           const C* __restrict__ out3, double2* __restrict__ q,
                                                           double2* __restrict__ H1, double2* __restrict__ hg,
                                                           double2* __restrict__ conv00) {
  constexpr int N = S * S, XB = sq_xbuf<S>();
  extern __shared__ __align__(16) unsigned char sq_raw[];
  const SqLane<S> ln;
  // three line buffers per group; the transforms exchange through line 0's
  C* lb = reinterpret_cast<C*>(sq_raw) + (ln.warp * SqLane<S>::G + ln.gi) * 3 * XB;
  const int K1 = g.kx_max + 1, K = g.kx_max;
  const int pair = (blockIdx.x * kSqWarps + ln.warp) * SqLane<S>::G + ln.gi;
  const bool act = ln.live && pair < g.ny * K1;
  const int y = act ? pair / K1 : 0;
  const int kx = act ? pair - y * K1 : 0;
  C tw[S - 1];
  sq_twiddles<S>(tw, twtab, ln.t);
  // h1 and h2 first (parked in lines 1 and 2), h0 last (lands in line 0)
#pragma unroll 1
  for (int k = 0; k < 3; ++k) {
    const int f = (k + 1) % 3;
    const C* src = out3 + (((size_t)f * g.ny + y) * K1 + kx) * N + ln.t;
    C x[S];
#pragma unroll
    for (int m = 0; m < S; ++m) x[m] = act ? src[S * m] : cmake<C>(0, 0);
    sq_fft<S, false>(x, tw, lb, ln.t, ln.live);
    if (ln.live) {
#pragma unroll
      for (int m = 0; m < S; ++m) lb[f * XB + ln.t + S * m] = x[m];
    }
  }
  __syncwarp();
  if (!act) return;
  const double cf = g.c_fwd;
  auto getF = [&](int f, int kz) -> double2 {
    const C v = lb[f * XB + (kz >= 0 ? kz : N + kz)];
    return make_double2((double)v.x * cf, (double)v.y * cf);
  };
  // rows this group owns: kx itself; -kx for 1 <= kx < K; the -K slot when kx = K
  int rows[2];
  int nrows = 1;
  rows[0] = kx;
  if (kx >= 1 && kx < K) rows[nrows++] = g.mx - kx;
  if (kx == K) rows[nrows++] = K + 1;
  for (int i = ln.t; i < nrows * g.mz; i += S) {
    const int rr = i >= g.mz ? 1 : 0;
    const int iz = i - rr * g.mz;
    const int ix = rows[rr];
    int sx, sz;
    bool cj;
    truncation_source(g, ix, iz, sx, sz, cj);
    double2 h[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const double2 val = (sx >= 0) ? getF(f, sz) : cconj(getF(f, -sz));
      h[f] = cj ? cconj(val) : val;
    }
    write_terms(g, y, ix, iz, h[0], h[1], h[2], q, H1, hg, conv00);
  }
}

template <typename C, int S>
size_t zfwd_sq_smem() {
  return sizeof(C) * (size_t)kSqWarps * SqLane<S>::G * 3 * sq_xbuf<S>();
}

// ---------------------------------------------------------------------------
// x pass with the products
// ---------------------------------------------------------------------------
// Shared-memory layout of the x pass, chosen so that every 64-bit request is
// served at the minimum number of wavefronts:
//   input tile [field][zl][kx], row stride KP: the staging copies (8 z columns
//     x 2 rows per half-warp) need KP = 2 mod 16 when ZC = 8; with more columns
//     per block an odd KP;
//   output tile [row][zl] with the 8 z columns of a row swizzled by
//     (row / 2) mod 8: the lanes of a group write 14 consecutive rows of one
//     column, the store reads 2 rows of 8 columns per half-warp;
//   twiddles lane-major (sq_tw_stride).
template <int ZC>
__host__ __device__ __forceinline__ int xsq_kp(int k1) {
  return ZC == 8 ? k1 + ((2 - k1) % 16 + 16) % 16 : k1 | 1;
}

template <typename C, int S>
struct XmidSq {
  static constexpr int G = SqLane<S>::G;
  static constexpr int ZC = kSqWarps * G;  // z columns per block
  static __host__ __device__ int kp(int k1) { return xsq_kp<ZC>(k1); }
  static constexpr int twn = (S - 1) * sq_tw_stride(S);  // twiddle table entries
  static size_t smem(const Geo& g, int nfields) {
    const int K1 = g.kx_max + 1;
    return sizeof(C) * ((size_t)nfields * ZC * kp(K1) + 3 * (size_t)K1 * ZC + (size_t)kSqWarps * G * sq_xbuf<S>() +
                        (size_t)twn);
  }
};

// slot of (row, z column) in the output tile
template <int ZC>
__device__ __forceinline__ int xsq_oslot(int row, int zl) {
  return ZC == 8 ? row * 8 + (zl ^ ((row >> 1) & 7)) : row * ZC + zl;
}

// Block-wide: the lane-major twiddle table from the table w_N^e, e = 0..N-1.
template <typename C, int S>
__device__ __forceinline__ void xsq_twiddle_table(C* stab, const C* __restrict__ twtab) {
  constexpr int TS = sq_tw_stride(S);
  for (int e = threadIdx.x; e < XmidSq<C, S>::twn; e += blockDim.x) {
    const int j = e / TS + 1, t = e - (j - 1) * TS;
    stab[e] = t < S ? twtab[t * j] : cmake<C>(0, 0);
  }
}

// 8- or 16-byte asynchronous copy global -> shared (zero fill when !ok)
template <typename C>
__device__ __forceinline__ void cp_async_elem(C* smem, const C* gmem, bool ok) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if constexpr (sizeof(C) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(ok ? 8 : 0));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(ok ? 16 : 0));
}

// Block-wide: start asynchronous copies of the input tile [f][zl][kx]
// (kx >= 0) of nfields fields; the caller waits (cp_async_wait<0>) and syncs.
template <typename C, int ZC>
__device__ __forceinline__ void xsq_stage_tile(const Geo& g, const C* __restrict__ inter, C* tile, int nfields,
                                               int y, int z0) {
  constexpr int RSTEP = kSqWarps * 32 / ZC;  // tile rows per pass of the block
  const int K1 = g.kx_max + 1, KP = xsq_kp<ZC>(K1);
  if (threadIdx.x < RSTEP * ZC) {
    const int zl = threadIdx.x % ZC;
    const int z = z0 + zl;
    const bool zok = z < g.pz;
    const C* base = inter + (size_t)y * K1 * g.pz + (zok ? z : 0);
    const size_t fstride = (size_t)g.ny * K1 * g.pz;
    int row = threadIdx.x / ZC;
    int f = row / K1, kx = row - (row / K1) * K1;
    for (; row < nfields * K1; row += RSTEP) {
      cp_async_elem(tile + (f * ZC + zl) * KP + kx, base + f * fstride + (size_t)kx * g.pz, zok);
      kx += RSTEP;
      while (kx >= K1) {
        kx -= K1;
        ++f;
      }
    }
  }
  cp_async_commit();
}

// Packed line a + i b of the column's fields (fa, fb), x-derivatives on request,
// at positions t + S m (same packing as fill_pair).
template <typename C, int S>
__device__ __forceinline__ void xsq_fill(const Geo& g, const C* tile, int zl, int t, bool live, C* x, int fa,
                                         bool dxa, int fb, bool dxb) {
  using Rl = typename real_of<C>::type;
  constexpr int N = S * S, ZC = XmidSq<C, S>::ZC;
  const int K = g.kx_max, KP = XmidSq<C, S>::kp(K + 1);
  const C* ta = tile + (fa * ZC + zl) * KP;
  const C* tb = tile + (fb * ZC + zl) * KP;
  // K < N / 2, so positions below N / 2 can only be kx >= 0 modes and those
  // above only kx < 0 modes: after unrolling, each m but a straddling one
  // needs one bound check and no select of the packing
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const int p = t + S * m;
    const bool below = S * m + S - 1 < N / 2, above = S * m >= N / 2;
    const bool lo = !above && p <= K, hi = !below && p >= N - K;
    C out = cmake<C>(0, 0);
    if (live && (lo || hi)) {
      const int kx = below ? p : above ? N - p : lo ? p : N - p;
      C A = ta[kx], B = tb[kx];
      const Rl k = (Rl)(kx * g.ax);
      if (dxa) A = cmul_ik(A, k);
      if (dxb) B = cmul_ik(B, k);
      if (m == 0 && p == 0) out = cmake<C>(A.x, B.x);
      else if (below || (!above && lo)) out = cmake<C>(A.x - B.y, A.y + B.x);
      else out = cmake<C>(A.x + B.y, B.x - A.y);
    }
    x[m] = out;
  }
}

// Forward transforms of (h0 + i h1) and (h2 + 0 i) of the column, kx >= 0
// outputs to the block's output tile [f][kx][zl].
template <typename C, int S>
__device__ __forceinline__ void xsq_forward(const Geo& g, const C* tab, C* xb, C* otile, int zl, int t, bool live,
                                            C* z01, C* z2) {
  using Rl = typename real_of<C>::type;
  constexpr int N = S * S, ZC = XmidSq<C, S>::ZC;
  const int K = g.kx_max, K1 = K + 1;
  sq_fft_tab<S, false>(z01, tab, xb, t, live);
  sq_fft_tab<S, false>(z2, tab, xb, t, live);
  if (live) {
#pragma unroll
    for (int m = 0; m < S; ++m) {
      xb[t + S * m] = z01[m];
      const int p = t + S * m;
      if (p <= K) otile[xsq_oslot<ZC>(2 * K1 + p, zl)] = z2[m];
    }
  }
  __syncwarp();
  if (live) {
    const Rl half = (Rl)0.5;
    for (int kx = t; kx <= K; kx += S) {
      const C a = xb[kx];
      const C b = xb[kx == 0 ? 0 : N - kx];
      // H0 = (Z[k] + conj Z[-k]) / 2, H1 = (Z[k] - conj Z[-k]) / (2 i)
      otile[xsq_oslot<ZC>(0 * K1 + kx, zl)] = cmake<C>(half * (a.x + b.x), half * (a.y - b.y));
      otile[xsq_oslot<ZC>(1 * K1 + kx, zl)] = cmake<C>(half * (a.y + b.y), -half * (a.x - b.x));
    }
  }
}

// Block-wide: coalesced store of the output tile.
template <typename C, int ZC>
__device__ __forceinline__ void xsq_store(const Geo& g, const C* otile, C* __restrict__ out3, int y, int z0) {
  constexpr int RSTEP = kSqWarps * 32 / ZC;
  const int K1 = g.kx_max + 1;
  if (threadIdx.x >= RSTEP * ZC) return;
  const int zl = threadIdx.x % ZC;
  const int z = z0 + zl;
  if (z >= g.pz) return;
  C* base = out3 + (size_t)y * K1 * g.pz + z;
  const size_t fstride = (size_t)g.ny * K1 * g.pz;
  int row = threadIdx.x / ZC;
  int f = row / K1, kx = row - (row / K1) * K1;
  for (; row < 3 * K1; row += RSTEP) {
    base[f * fstride + (size_t)kx * g.pz] = otile[xsq_oslot<ZC>(row, zl)];
    kx += RSTEP;
    while (kx >= K1) {
      kx -= K1;
      ++f;
    }
  }
}

// Resident blocks per SM the FP32 x pass is compiled for (registers capped at
// 168 per lane: a little spilling, 12 warps per SM instead of 8).
template <typename C>
constexpr int xsq_min_blocks() {
  return sizeof(C) == sizeof(float2) ? 3 : 1;
}

// NS / perturbation products, as in k_xmid:
//   hel_i = -lam (u . grad) u_i + lam/2 (div u) u_i - U d_x u_i - delta_i0 (v U' - (div u) U / 2)
template <typename C, int S>
__global__ void __launch_bounds__(kSqWarps * 32, xsq_min_blocks<C>()) k_xmid_sq(Geo g, const C* __restrict__ twtab,
                                                           const C* __restrict__ inter, C* __restrict__ out3,
                                                           const double* __restrict__ ubase,
                                                           const double* __restrict__ dubase, double lam_d) {
  using Rl = typename real_of<C>::type;
  constexpr int G = SqLane<S>::G, ZC = XmidSq<C, S>::ZC, XB = sq_xbuf<S>();
  extern __shared__ __align__(16) unsigned char sq_raw[];
  const int K1 = g.kx_max + 1, KP = XmidSq<C, S>::kp(K1);
  C* tile = reinterpret_cast<C*>(sq_raw);
  C* otile = tile + kZinvLines * ZC * KP;
  const SqLane<S> ln;
  C* xb = otile + 3 * K1 * ZC + (ln.warp * G + ln.gi) * XB;
  const int z0 = blockIdx.x * ZC, y = blockIdx.y;
  const int zl = ln.warp * G + ln.gi;
  const Rl ub = ubase ? (Rl)ubase[y / g.nb] : (Rl)0;
  const Rl dub = dubase ? (Rl)dubase[y / g.nb] : (Rl)0;
  const Rl c = (Rl)g.c_inv, lam = (Rl)lam_d, half = (Rl)0.5;
  xsq_stage_tile<C, ZC>(g, inter, tile, kZinvLines, y, z0);
  // twiddle table in shared memory (read by stage 1 of every transform)
  C* stab = otile + 3 * K1 * ZC + kSqWarps * G * XB;
  xsq_twiddle_table<C, S>(stab, twtab);
  cp_async_wait<0>();
  __syncthreads();
  const bool live = ln.live;
  const int t = ln.t;
  // intermediate: 0 u, 1 v, 2 w, 3 du/dy, 4 dv/dy, 5 dw/dy, 6 du/dz, 7 dv/dz, 8 dw/dz
  Rl U[S], V[S], W[S], DIV[S], A0[S], A1[S], A2[S];
  C x[S];
  xsq_fill<C, S>(g, tile, zl, t, live, x, 0, false, 1, false);  // (u, v)
  sq_fft_tab<S, true>(x, stab, xb, t, live);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    U[m] = x[m].x * c;
    V[m] = x[m].y * c;
  }
  xsq_fill<C, S>(g, tile, zl, t, live, x, 2, false, 0, true);  // (w, du/dx)
  sq_fft_tab<S, true>(x, stab, xb, t, live);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    W[m] = x[m].x * c;
    const Rl dxu = x[m].y * c;
    DIV[m] = dxu;
    A0[m] = lam * U[m] * dxu + ub * dxu;
  }
  xsq_fill<C, S>(g, tile, zl, t, live, x, 1, true, 2, true);  // (dv/dx, dw/dx)
  sq_fft_tab<S, true>(x, stab, xb, t, live);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const Rl dxv = x[m].x * c, dxw = x[m].y * c;
    A1[m] = lam * U[m] * dxv + ub * dxv;
    A2[m] = lam * U[m] * dxw + ub * dxw;
  }
  xsq_fill<C, S>(g, tile, zl, t, live, x, 4, false, 8, false);  // (dv/dy, dw/dz)
  sq_fft_tab<S, true>(x, stab, xb, t, live);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const Rl dyv = x[m].x * c, dzw = x[m].y * c;
    DIV[m] += dyv + dzw;
    A1[m] += lam * V[m] * dyv;
    A2[m] += lam * W[m] * dzw;
  }
  xsq_fill<C, S>(g, tile, zl, t, live, x, 3, false, 5, false);  // (du/dy, dw/dy)
  sq_fft_tab<S, true>(x, stab, xb, t, live);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const Rl dyu = x[m].x * c, dyw = x[m].y * c;
    A0[m] += lam * V[m] * dyu;
    A2[m] += lam * V[m] * dyw;
  }
  xsq_fill<C, S>(g, tile, zl, t, live, x, 6, false, 7, false);  // (du/dz, dv/dz)
  sq_fft_tab<S, true>(x, stab, xb, t, live);
  C z2[S];
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const Rl dzu = x[m].x * c, dzv = x[m].y * c;
    const Rl a0 = A0[m] + lam * W[m] * dzu;
    const Rl a1 = A1[m] + lam * W[m] * dzv;
    const Rl d = DIV[m];
    const Rl h0 = -a0 + half * lam * d * U[m] - V[m] * dub + half * d * ub;
    const Rl h1 = -a1 + half * lam * d * V[m];
    const Rl h2 = -A2[m] + half * lam * d * W[m];
    x[m] = cmake<C>(h0, h1);
    z2[m] = cmake<C>(h2, (Rl)0);
  }
  xsq_forward<C, S>(g, stab, xb, otile, zl, t, live && z0 + zl < g.pz, x, z2);
  __syncthreads();
  xsq_store<C, ZC>(g, otile, out3, y, z0);
}

// Adjoint products, as in k_xmid_dual (lam = 1; dual v, frozen forward u,
// base U(y) e_x, Ut = U + u):
//   hel_i = -(Ut . grad) v_i + sum_j v_j d_i Ut_j + [(div u) v_i + (div v) Ut_i] / 4
// Intermediate lines 0..8 hold v (v, dv/dy, dv/dz), 9..17 the same for u.
template <typename C, int S>
__global__ void __launch_bounds__(kSqWarps * 32) k_xmid_dual_sq(Geo g, const C* __restrict__ twtab,
                                                                const C* __restrict__ inter, C* __restrict__ out3,
                                                                const double* __restrict__ ubase,
                                                                const double* __restrict__ dubase) {
  using Rl = typename real_of<C>::type;
  constexpr int G = SqLane<S>::G, ZC = XmidSq<C, S>::ZC, XB = sq_xbuf<S>();
  extern __shared__ __align__(16) unsigned char sq_raw[];
  const int K1 = g.kx_max + 1, KP = XmidSq<C, S>::kp(K1);
  C* tile = reinterpret_cast<C*>(sq_raw);
  C* otile = tile + 2 * kZinvLines * ZC * KP;
  const SqLane<S> ln;
  C* xb = otile + 3 * K1 * ZC + (ln.warp * G + ln.gi) * XB;
  const int z0 = blockIdx.x * ZC, y = blockIdx.y;
  const int zl = ln.warp * G + ln.gi;
  const Rl ub = (Rl)ubase[y / g.nb];
  const Rl dub = (Rl)dubase[y / g.nb];
  const Rl c = (Rl)g.c_inv, q4 = (Rl)0.25;
  xsq_stage_tile<C, ZC>(g, inter, tile, 2 * kZinvLines, y, z0);
  // twiddle table in shared memory (read by stage 1 of every transform)
  C* stab = otile + 3 * K1 * ZC + kSqWarps * G * XB;
  xsq_twiddle_table<C, S>(stab, twtab);
  cp_async_wait<0>();
  __syncthreads();
  const bool live = ln.live;
  const int t = ln.t;
  Rl V0[S], V1[S], V2[S], U0[S], U1[S], U2[S], A0[S], A1[S], A2[S], DV[S], DU[S];
  C x[S];
#define JSD_LINE(fa, dxa, fb, dxb)                           \
  xsq_fill<C, S>(g, tile, zl, t, live, x, fa, dxa, fb, dxb); \
  sq_fft_tab<S, true>(x, stab, xb, t, live);
#define JSD_EACH(body)                                       \
  _Pragma("unroll") for (int m = 0; m < S; ++m) {            \
    const Rl pa = x[m].x * c, pb = x[m].y * c;               \
    body                                                     \
  }
  JSD_LINE(0, false, 1, false)  // (v0, v1)
  JSD_EACH(V0[m] = pa; V1[m] = pb;)
  JSD_LINE(2, false, 9, false)  // (v2, u0)
  JSD_EACH(V2[m] = pa; U0[m] = pb;)
  JSD_LINE(10, false, 11, false)  // (u1, u2)
  JSD_EACH(U1[m] = pa; U2[m] = pb;)
  JSD_LINE(0, true, 1, true)  // (dv0/dx, dv1/dx)
  JSD_EACH(const Rl ut = ub + U0[m]; A0[m] = -ut * pa; A1[m] = -ut * pb; DV[m] = pa;)
  JSD_LINE(2, true, 3, false)  // (dv2/dx, dv0/dy)
  JSD_EACH(A2[m] = -(ub + U0[m]) * pa; A0[m] -= U1[m] * pb;)
  JSD_LINE(4, false, 5, false)  // (dv1/dy, dv2/dy)
  JSD_EACH(A1[m] -= U1[m] * pa; A2[m] -= U1[m] * pb; DV[m] += pa;)
  JSD_LINE(6, false, 7, false)  // (dv0/dz, dv1/dz)
  JSD_EACH(A0[m] -= U2[m] * pa; A1[m] -= U2[m] * pb;)
  JSD_LINE(8, false, 9, true)  // (dv2/dz, du0/dx)
  JSD_EACH(A2[m] -= U2[m] * pa; DV[m] += pa; A0[m] += V0[m] * pb; DU[m] = pb;)
  JSD_LINE(10, true, 11, true)  // (du1/dx, du2/dx)
  JSD_EACH(A0[m] += V1[m] * pa + V2[m] * pb;)
  JSD_LINE(12, false, 13, false)  // (du0/dy, du1/dy)
  JSD_EACH(A1[m] += V0[m] * pa + V1[m] * pb; DU[m] += pb;)
  JSD_LINE(14, false, 15, false)  // (du2/dy, du0/dz)
  JSD_EACH(A1[m] += V2[m] * pa; A2[m] += V0[m] * pb;)
  JSD_LINE(16, false, 17, false)  // (du1/dz, du2/dz)
  C z2[S];
  JSD_EACH(
      A2[m] += V1[m] * pa + V2[m] * pb; DU[m] += pb; const Rl du = DU[m]; const Rl dv = DV[m];
      const Rl h0 = A0[m] + q4 * du * V0[m] + q4 * dv * (ub + U0[m]);
      const Rl h1 = A1[m] + dub * V0[m] + q4 * du * V1[m] + q4 * dv * U1[m];
      const Rl h2 = A2[m] + q4 * du * V2[m] + q4 * dv * U2[m]; x[m] = cmake<C>(h0, h1); z2[m] = cmake<C>(h2, (Rl)0);)
#undef JSD_LINE
#undef JSD_EACH
  xsq_forward<C, S>(g, stab, xb, otile, zl, t, live && z0 + zl < g.pz, x, z2);
  __syncthreads();
  xsq_store<C, ZC>(g, otile, out3, y, z0);
}

// ---------------------------------------------------------------------------
// x pass, half-split lanes (even S): a z column's lines on 2 S lanes, H = S / 2
// points per lane (sq2_fft). Half the registers per lane of k_xmid_sq, so the
// FP64 products fit without spilling.
// ---------------------------------------------------------------------------
template <int S>
struct SqLane2 {
  static constexpr int H = S / 2, L = 2 * S, G = 32 / L;  // lines per warp
  int warp, gi, t, h, partner;
  bool live;
  __device__ __forceinline__ SqLane2() {
    const int lane = threadIdx.x & 31;
    warp = threadIdx.x >> 5;
    gi = lane / L;
    const int r = lane - gi * L;
    h = r / S;
    t = r - h * S;
    live = gi < G;
    if (!live) {
      gi = 0;
      h = 0;
      t = 0;
    }
    partner = live ? (h ? lane - S : lane + S) : lane;
  }
};

template <typename C, int S>
struct XmidH2 {
  static constexpr int G = SqLane2<S>::G;
  static constexpr int ZC = kSqWarps * G;
  static size_t smem(const Geo& g, int nfields) {
    const int K1 = g.kx_max + 1;
    return sizeof(C) * ((size_t)nfields * ZC * (K1 | 1) + 3 * (size_t)K1 * ZC + (size_t)kSqWarps * G * sq_xbuf<S>() +
                        (size_t)S * S);
  }
};

// packed line of fields (fa, fb) at this lane's positions t + S (2 j + h)
template <typename C, int S, int ZC>
__device__ __forceinline__ void xh2_fill(const Geo& g, const C* tile, int zl, int t, int h, bool live, C* x, int fa,
                                         bool dxa, int fb, bool dxb) {
  using Rl = typename real_of<C>::type;
  constexpr int N = S * S, H = S / 2;
  const int K = g.kx_max, KP = (K + 1) | 1;
  const C* ta = tile + (fa * ZC + zl) * KP;
  const C* tb = tile + (fb * ZC + zl) * KP;
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const int p = t + S * (2 * j + h);
    const bool lo = p <= K, hi = p >= N - K;
    C out = cmake<C>(0, 0);
    if (live && (lo || hi)) {
      const int kx = lo ? p : N - p;
      C A = ta[kx], B = tb[kx];
      const Rl k = (Rl)(kx * g.ax);
      if (dxa) A = cmul_ik(A, k);
      if (dxb) B = cmul_ik(B, k);
      if (p == 0) out = cmake<C>(A.x, B.x);
      else if (lo) out = cmake<C>(A.x - B.y, A.y + B.x);
      else out = cmake<C>(A.x + B.y, B.x - A.y);
    }
    x[j] = out;
  }
}

template <typename C, int S>
__global__ void __launch_bounds__(kSqWarps * 32) k_xmid_h2(Geo g, const C* __restrict__ twtab,
                                                           const C* __restrict__ inter, C* __restrict__ out3,
                                                           const double* __restrict__ ubase,
                                                           const double* __restrict__ dubase, double lam_d) {
  using Rl = typename real_of<C>::type;
  constexpr int N = S * S, H = S / 2, G = SqLane2<S>::G, ZC = XmidH2<C, S>::ZC, XB = sq_xbuf<S>();
  extern __shared__ __align__(16) unsigned char sq_raw[];
  const int K = g.kx_max, K1 = K + 1, KP = K1 | 1;
  C* tile = reinterpret_cast<C*>(sq_raw);
  C* otile = tile + kZinvLines * ZC * KP;
  const SqLane2<S> ln;
  C* xb = otile + 3 * K1 * ZC + (ln.warp * G + ln.gi) * XB;
  C* stab = otile + 3 * K1 * ZC + kSqWarps * G * XB;
  const int z0 = blockIdx.x * ZC, y = blockIdx.y;
  const int zl = ln.warp * G + ln.gi;
  const Rl ub = ubase ? (Rl)ubase[y / g.nb] : (Rl)0;
  const Rl dub = dubase ? (Rl)dubase[y / g.nb] : (Rl)0;
  const Rl c = (Rl)g.c_inv, lam = (Rl)lam_d, half = (Rl)0.5;
  xsq_stage_tile<C, ZC>(g, inter, tile, kZinvLines, y, z0);
  for (int e = threadIdx.x; e < N; e += blockDim.x) stab[e] = twtab[e];
  cp_async_wait<0>();
  __syncthreads();
  const bool live = ln.live;
  const int t = ln.t, h = ln.h, pr = ln.partner;
  Rl U[H], V[H], W[H], DIV[H], A0[H], A1[H], A2[H];
  C x[H];
  xh2_fill<C, S, ZC>(g, tile, zl, t, h, live, x, 0, false, 1, false);  // (u, v)
  sq2_fft<S, true>(x, stab, xb, t, h, pr, live);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    U[j] = x[j].x * c;
    V[j] = x[j].y * c;
  }
  xh2_fill<C, S, ZC>(g, tile, zl, t, h, live, x, 2, false, 0, true);  // (w, du/dx)
  sq2_fft<S, true>(x, stab, xb, t, h, pr, live);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    W[j] = x[j].x * c;
    const Rl dxu = x[j].y * c;
    DIV[j] = dxu;
    A0[j] = lam * U[j] * dxu + ub * dxu;
  }
  xh2_fill<C, S, ZC>(g, tile, zl, t, h, live, x, 1, true, 2, true);  // (dv/dx, dw/dx)
  sq2_fft<S, true>(x, stab, xb, t, h, pr, live);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const Rl dxv = x[j].x * c, dxw = x[j].y * c;
    A1[j] = lam * U[j] * dxv + ub * dxv;
    A2[j] = lam * U[j] * dxw + ub * dxw;
  }
  xh2_fill<C, S, ZC>(g, tile, zl, t, h, live, x, 4, false, 8, false);  // (dv/dy, dw/dz)
  sq2_fft<S, true>(x, stab, xb, t, h, pr, live);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const Rl dyv = x[j].x * c, dzw = x[j].y * c;
    DIV[j] += dyv + dzw;
    A1[j] += lam * V[j] * dyv;
    A2[j] += lam * W[j] * dzw;
  }
  xh2_fill<C, S, ZC>(g, tile, zl, t, h, live, x, 3, false, 5, false);  // (du/dy, dw/dy)
  sq2_fft<S, true>(x, stab, xb, t, h, pr, live);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const Rl dyu = x[j].x * c, dyw = x[j].y * c;
    A0[j] += lam * V[j] * dyu;
    A2[j] += lam * V[j] * dyw;
  }
  xh2_fill<C, S, ZC>(g, tile, zl, t, h, live, x, 6, false, 7, false);  // (du/dz, dv/dz)
  sq2_fft<S, true>(x, stab, xb, t, h, pr, live);
  C z2[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const Rl dzu = x[j].x * c, dzv = x[j].y * c;
    const Rl a0 = A0[j] + lam * W[j] * dzu;
    const Rl a1 = A1[j] + lam * W[j] * dzv;
    const Rl d = DIV[j];
    const Rl h0 = -a0 + half * lam * d * U[j] - V[j] * dub + half * d * ub;
    const Rl h1 = -a1 + half * lam * d * V[j];
    const Rl h2 = -A2[j] + half * lam * d * W[j];
    x[j] = cmake<C>(h0, h1);
    z2[j] = cmake<C>(h2, (Rl)0);
  }
  // forward transforms and the kx >= 0 outputs of the column
  const bool colok = live && z0 + zl < g.pz;
  sq2_fft<S, false>(x, stab, xb, t, h, pr, colok);
  sq2_fft<S, false>(z2, stab, xb, t, h, pr, colok);
  if (colok) {
#pragma unroll
    for (int j = 0; j < H; ++j) {
      const int p = t + S * (2 * j + h);
      xb[p] = x[j];
      if (p <= K) otile[(2 * K1 + p) * ZC + zl] = z2[j];
    }
  }
  __syncwarp();
  if (colok) {
    for (int kx = h * S + t; kx <= K; kx += 2 * S) {
      const C a = xb[kx];
      const C b = xb[kx == 0 ? 0 : N - kx];
      otile[xsq_oslot<ZC>(0 * K1 + kx, zl)] = cmake<C>(half * (a.x + b.x), half * (a.y - b.y));
      otile[xsq_oslot<ZC>(1 * K1 + kx, zl)] = cmake<C>(half * (a.y + b.y), -half * (a.x - b.x));
    }
  }
  __syncthreads();
  xsq_store<C, ZC>(g, otile, out3, y, z0);
}

}  // namespace jsd
