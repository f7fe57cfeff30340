// Register-resident FFTs of square length N = S * S, one line per group of S
// lanes of a warp.
//
// Four-step form with n = S n1 + n2 and k = k1 + S k2:
//   X[k1 + S k2] = sum_n2 w_S^(n2 k2) w_N^(n2 k1) [ sum_n1 x[S n1 + n2] w_S^(n1 k1) ]
// Lane t of a group holds the elements at positions t + S m (m = 0..S-1) of
// its line. Stage 1: lane t (= n2) takes the S-point DFT over m, multiplies
// entry k1 by w_N^(t k1) and writes it to row k1, column t of the group's
// exchange buffer; stage 2: lane t (= k1) reads row t and takes the S-point
// DFT over the columns. The result X[t + S k2] lands in register k2, so every
// lane holds the same positions of the output as of the input: pointwise work
// between an inverse and a forward transform stays in registers, and the only
// synchronisation is a __syncwarp around the exchange.
//
// S-point DFTs in registers: radices 2, 3, 4, 5, 7, 8 directly (jsd_fft.cuh),
// composite S with coprime factors by the prime-factor (Good-Thomas) mapping,
// which needs no twiddles: n = (B n1 + A n2) mod S, k = (B (B^-1 mod A) k1 +
// A (A^-1 mod B) k2) mod S for S = A B.
#pragma once

#include "jsd_common.cuh"
#include "jsd_fft.cuh"

namespace jsd {

__host__ __device__ constexpr int sq_inv_mod(int a, int m) {
  for (int x = 1; x < m; ++x)
    if ((a * x) % m == 1) return x;
  return 1;
}

// first factor A of the prime-factor split used for S (0: S is a base radix)
__host__ __device__ constexpr int sq_split(int s) {
  return s == 6 ? 2 : s == 10 ? 2 : s == 12 ? 4 : s == 14 ? 2 : s == 15 ? 3 : s == 20 ? 4 : s == 21 ? 3
       : s == 24 ? 8 : s == 28 ? 4 : s == 30 ? 2 : 0;
}

__host__ __device__ constexpr bool sq_supported(int s) {
  return s == 2 || s == 3 || s == 4 || s == 5 || s == 7 || s == 8 || sq_split(s) != 0;
}

template <int R, bool INV, typename C>
__host__ __device__ __forceinline__ void dft_reg(C* x);

template <int A, int B, bool INV, typename C>
__host__ __device__ __forceinline__ void dft_pfa(C* x) {
  constexpr int N = A * B;
  constexpr int binv = sq_inv_mod(B % A, A);
  constexpr int ainv = sq_inv_mod(A % B, B);
  C t[N];
#pragma unroll
  for (int n1 = 0; n1 < A; ++n1)
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) t[n1 * B + n2] = x[(B * n1 + A * n2) % N];
#pragma unroll
  for (int n2 = 0; n2 < B; ++n2) {
    C a[A];
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) a[n1] = t[n1 * B + n2];
    dft_reg<A, INV>(a);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) t[k1 * B + n2] = a[k1];
  }
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    C b[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) b[n2] = t[k1 * B + n2];
    dft_reg<B, INV>(b);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) x[(B * binv * k1 + A * ainv * k2) % N] = b[k2];
  }
}

template <int R, bool INV, typename C>
__host__ __device__ __forceinline__ void dft_reg(C* x) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<INV>(x);
  } else if constexpr (R == 4) {
    dft4<INV>(x);
  } else if constexpr (R == 8) {
    dft8<INV>(x);
  } else if constexpr (R == 3 || R == 5 || R == 7) {
    dft_odd<R, INV>(x);
  } else {
    static_assert(sq_split(R) != 0, "unsupported register DFT length");
    dft_pfa<sq_split(R), R / sq_split(R), INV>(x);
  }
}

// Exchange-buffer elements per group (rows padded to S + 1 against bank conflicts).
template <int S>
__host__ __device__ constexpr int sq_xbuf() {
  return S * (S + 1);
}

// Stage 1 of a transform of the line held by the S lanes of a group (t =
// lane in the group): x[m] = element t + S m on entry; the S-point DFT over m,
// times w_N^(t j), goes to row j, column t of the group's exchange buffer xb.
// tw[j - 1] = w_N^(t j) with the forward sign, j = 1..S-1.
template <int S, bool INV, typename C>
__host__ __device__ __forceinline__ void sq_stage1(C* x, const C* tw, C* xb, int t) {
  dft_reg<S, INV>(x);
#pragma unroll
  for (int j = 1; j < S; ++j) {
    C w = tw[j - 1];
    if (INV) w.y = -w.y;
    x[j] = cmul(x[j], w);
  }
#pragma unroll
  for (int j = 0; j < S; ++j) xb[j * (S + 1) + t] = x[j];
}

// Stage 2: lane t reads row t and transforms it; x[m] = X[t + S m] on exit.
template <int S, bool INV, typename C>
__host__ __device__ __forceinline__ void sq_stage2(C* x, const C* xb, int t) {
#pragma unroll
  for (int j = 0; j < S; ++j) x[j] = xb[t * (S + 1) + j];
  dft_reg<S, INV>(x);
}

// The whole transform. Every lane of the warp must call it, since the exchange
// is synchronised warp-wide; lanes outside any group pass live = false.
template <int S, bool INV, typename C>
__device__ __forceinline__ void sq_fft(C* x, const C* tw, C* xb, int t, bool live) {
  if (live) sq_stage1<S, INV>(x, tw, xb, t);
  __syncwarp();
  if (live) sq_stage2<S, INV>(x, xb, t);
  __syncwarp();
}

// Row stride of the lane-major twiddle table: entry (j, t) = w_N^(t j) sits at
// (j - 1) * stride + t, so the lanes of a group read consecutive entries.
__host__ __device__ constexpr int sq_tw_stride(int s) {
  return s <= 16 ? 16 : 32;
}

// sq_fft with the twiddles read from the lane-major table (sq_tw_stride;
// typically in shared memory) instead of registers.
template <int S, bool INV, typename C>
__device__ __forceinline__ void sq_fft_tab(C* x, const C* tab, C* xb, int t, bool live) {
  constexpr int TS = sq_tw_stride(S);
  if (live) {
    dft_reg<S, INV>(x);
#pragma unroll
    for (int j = 1; j < S; ++j) {
      C w = tab[(j - 1) * TS + t];
      if (INV) w.y = -w.y;
      x[j] = cmul(x[j], w);
    }
#pragma unroll
    for (int j = 0; j < S; ++j) xb[j * (S + 1) + t] = x[j];
  }
  __syncwarp();
  if (live) sq_stage2<S, INV>(x, xb, t);
  __syncwarp();
}

// Half-split form for even S = 2H: a line on 2S lanes, lane (t, h) holding
// the H elements at positions t + S (2 j + h), j = 0..H-1.
//   stage 1, decimation in time over m = 2 j + h: lane h transforms its own
//     H values (E for h = 0, O for h = 1), swaps them with its partner lane
//     (same t, other h), and forms Y[h H + k] = E[k] +- w_S^k O[k], times
//     w_N^(t (h H + k)), into the exchange buffer;
//   stage 2, decimation in frequency: lane (t, h) reads row t and forms
//     c[n] = b[n] + b[n+H] (h = 0) or (b[n] - b[n+H]) w_S^n (h = 1), whose
//     H-point DFT is X[t + S (2 j + h)].
// Input and output positions of a lane coincide, as in sq_fft. tab = w_N^e.
// Stage-1 butterfly of the half-split form for one k: own = this lane's
// H-point DFT value at k, other = the partner lane's.
template <int S, bool INV, typename C>
__host__ __device__ __forceinline__ C sq2_butterfly(C own, C other, int k, const C* tab, int t, int h) {
  constexpr int H = S / 2;
  const C E = h ? other : own;
  C O = h ? own : other;
  C w = tab[S * k];
  if (INV) w.y = -w.y;
  O = cmul(O, w);
  const C y = h ? csub(E, O) : cadd(E, O);
  C tw = tab[t * (h * H + k)];
  if (INV) tw.y = -tw.y;
  return cmul(y, tw);
}

// Stage 2 of the half-split form: read row t of the exchange buffer, combine
// for output parity h, H-point DFT; x[j] = X[t + S (2 j + h)] on exit.
template <int S, bool INV, typename C>
__host__ __device__ __forceinline__ void sq2_stage2(C* x, const C* xb, const C* tab, int t, int h) {
  constexpr int H = S / 2;
#pragma unroll
  for (int n = 0; n < H; ++n) {
    const C b0 = xb[t * (S + 1) + n], b1 = xb[t * (S + 1) + n + H];
    if (h) {
      C w = tab[S * n];
      if (INV) w.y = -w.y;
      x[n] = cmul(csub(b0, b1), w);
    } else {
      x[n] = cadd(b0, b1);
    }
  }
  dft_reg<H, INV>(x);
}

template <int S, bool INV, typename C>
__device__ __forceinline__ void sq2_fft(C* x, const C* tab, C* xb, int t, int h, int partner, bool live) {
  constexpr int H = S / 2;
  static_assert(2 * H == S, "half-split transform needs an even side");
  dft_reg<H, INV>(x);
#pragma unroll
  for (int k = 0; k < H; ++k) {
    C o;
    o.x = __shfl_sync(0xffffffffu, x[k].x, partner);
    o.y = __shfl_sync(0xffffffffu, x[k].y, partner);
    x[k] = sq2_butterfly<S, INV>(x[k], o, k, tab, t, h);
  }
  if (live) {
#pragma unroll
    for (int k = 0; k < H; ++k) xb[(h * H + k) * (S + 1) + t] = x[k];
  }
  __syncwarp();
  if (live) sq2_stage2<S, INV>(x, xb, tab, t, h);
  __syncwarp();
}

// Lane t's twiddles w_N^(t j), j = 1..S-1, from the table w_N^e, e = 0..N-1.
template <int S, typename C>
__host__ __device__ __forceinline__ void sq_twiddles(C* tw, const C* __restrict__ table, int t) {
#pragma unroll
  for (int j = 1; j < S; ++j) tw[j - 1] = table[t * j];
}

}  // namespace jsd
