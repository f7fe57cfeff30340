// Batched mixed-radix FFT of complex-double lines held in shared memory.
//
// Stockham autosort formulation: pass p with radix r and sub-transform length
// Ls reads x[j + t*n/r] (t < r), multiplies by w^(t*k) with k = j mod Ls and
// w = exp(-+2 pi i / (Ls r)), applies an r-point DFT and writes to
// (j / Ls) * Ls * r + k + t * Ls. Passes ping-pong between two buffers, so the
// result ends in whichever buffer the last pass wrote; the routine returns it.
// Radices 2, 3, 4, 5, 7 and 8 are supported. The twiddle table holds, for each
// pass, Ls * (r - 1) forward twiddles exp(-2 pi i t k / (Ls r)) in (k, t)
// order; the inverse uses their conjugates. Transforms are unnormalised.
#pragma once

#include "jsd_common.cuh"

namespace jsd {

constexpr int kMaxFftPasses = 12;

struct FftDesc {
  int n;
  int passes;
  int radix[kMaxFftPasses];
  int ls[kMaxFftPasses];
  int twoff[kMaxFftPasses];
};

// Lines are stored with one padding slot after every 32 complex elements so
// the strided Stockham writes spread over all shared-memory banks.
__host__ __device__ __forceinline__ int fpad(int i) { return i + (i >> 5); }
__host__ __device__ __forceinline__ int fline(int n) { return n + (n >> 5) + 1; }

// cos(2 pi m / R) and sin(2 pi m / R) for R = 3, 5, 7 (m = 0..R-1)
__host__ __device__ __forceinline__ void root_table(int r, int m, double& c, double& s) {
  if (r == 3) {
    const double C[3] = {1.0, -0.5, -0.5};
    const double S[3] = {0.0, 0.86602540378443864676, -0.86602540378443864676};
    c = C[m]; s = S[m];
  } else if (r == 5) {
    const double C[5] = {1.0, 0.30901699437494742410, -0.80901699437494742410,
                         -0.80901699437494742410, 0.30901699437494742410};
    const double S[5] = {0.0, 0.95105651629515357212, 0.58778525229247312917,
                         -0.58778525229247312917, -0.95105651629515357212};
    c = C[m]; s = S[m];
  } else {  // 7
    const double C[7] = {1.0, 0.62348980185873353053, -0.22252093395631440429, -0.90096886790241912624,
                         -0.90096886790241912624, -0.22252093395631440429, 0.62348980185873353053};
    const double S[7] = {0.0, 0.78183148246802980871, 0.97492791218182360702, 0.43388373911755812048,
                         -0.43388373911755812048, -0.97492791218182360702, -0.78183148246802980871};
    c = C[m]; s = S[m];
  }
}

// Odd-radix DFT in conjugate-pair form: with a_t = x_t + x_{R-t} and
// b_t = x_t - x_{R-t} (t = 1..h, h = (R-1)/2),
//   y[q]   = x_0 + sum_t a_t cos(2 pi q t / R) -+ i sum_t b_t sin(2 pi q t / R)
//   y[R-q] = x_0 + sum_t a_t cos(2 pi q t / R) +- i sum_t b_t sin(2 pi q t / R)
// (upper signs forward), h^2 complex-by-real products per half instead of R^2.
template <int R, bool INV, typename C>
__host__ __device__ __forceinline__ void dft_odd(C* x) {
  using Rl = typename real_of<C>::type;
  constexpr int H = (R - 1) / 2;
  C a[H], b[H];
  C y0 = x[0];
#pragma unroll
  for (int t = 1; t <= H; ++t) {
    a[t - 1] = cadd(x[t], x[R - t]);
    b[t - 1] = csub(x[t], x[R - t]);
    y0 = cadd(y0, a[t - 1]);
  }
  C y[R];
  y[0] = y0;
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    C re = x[0], im = cmake<C>(0, 0);
#pragma unroll
    for (int t = 1; t <= H; ++t) {
      double cd, sd;
      root_table(R, (q * t) % R, cd, sd);
      const Rl c = (Rl)cd, sn = (Rl)sd;
      re.x += a[t - 1].x * c;
      re.y += a[t - 1].y * c;
      im.x += b[t - 1].x * sn;
      im.y += b[t - 1].y * sn;
    }
    // i * im = (-im.y, im.x)
    const C iim = cmake<C>(-im.y, im.x);
    y[q] = INV ? cadd(re, iim) : csub(re, iim);
    y[R - q] = INV ? csub(re, iim) : cadd(re, iim);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) x[q] = y[q];
}

template <bool INV, typename C>
__host__ __device__ __forceinline__ void dft2(C* x) {
  const C a = x[0], b = x[1];
  x[0] = cadd(a, b);
  x[1] = csub(a, b);
}

// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C>
__host__ __device__ __forceinline__ C rot90(C a) {
  return INV ? cmake<C>(-a.y, a.x) : cmake<C>(a.y, -a.x);
}

template <bool INV, typename C>
__host__ __device__ __forceinline__ void dft4(C* x) {
  const C s02 = cadd(x[0], x[2]), d02 = csub(x[0], x[2]);
  const C s13 = cadd(x[1], x[3]), d13 = rot90<INV>(csub(x[1], x[3]));
  x[0] = cadd(s02, s13);
  x[2] = csub(s02, s13);
  x[1] = cadd(d02, d13);
  x[3] = csub(d02, d13);
}

template <bool INV, typename C>
__host__ __device__ __forceinline__ void dft8(C* x) {
  using Rl = typename real_of<C>::type;
  const Rl h = (Rl)0.70710678118654752440;
  C e[4] = {x[0], x[2], x[4], x[6]};
  C o[4] = {x[1], x[3], x[5], x[7]};
  dft4<INV>(e);
  dft4<INV>(o);
  // twiddles exp(-+2 pi i m / 8), m = 0..3
  const C o1 = INV ? cmake<C>(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                   : cmake<C>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
  const C o2 = rot90<INV>(o[2]);
  const C o3 = INV ? cmake<C>(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                   : cmake<C>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
  x[0] = cadd(e[0], o[0]);
  x[4] = csub(e[0], o[0]);
  x[1] = cadd(e[1], o1);
  x[5] = csub(e[1], o1);
  x[2] = cadd(e[2], o2);
  x[6] = csub(e[2], o2);
  x[3] = cadd(e[3], o3);
  x[7] = csub(e[3], o3);
}

template <int R, bool INV, typename C>
__device__ __forceinline__ void fft_pass(const C* __restrict__ src, C* __restrict__ dst, int nlines, int n, int ls,
                                         const C* __restrict__ tw) {
  const int m = n / R;
  const int total = nlines * m;
  const int stride = fline(n);
  for (int task = threadIdx.x; task < total; task += blockDim.x) {
    const int l = task / m;
    const int j = task - l * m;
    const int k = j % ls;
    const C* s = src + (size_t)l * stride;
    C x[R];
#pragma unroll
    for (int t = 0; t < R; ++t) x[t] = s[fpad(j + t * m)];
    if (ls > 1) {
#pragma unroll
      for (int t = 1; t < R; ++t) {
        C w = tw[k * (R - 1) + (t - 1)];
        if (INV) w.y = -w.y;
        x[t] = cmul(x[t], w);
      }
    }
    if constexpr (R == 2) dft2<INV>(x);
    else if constexpr (R == 4) dft4<INV>(x);
    else if constexpr (R == 8) dft8<INV>(x);
    else dft_odd<R, INV>(x);
    C* o = dst + (size_t)l * stride;
    const int base = (j / ls) * ls * R + k;
#pragma unroll
    for (int t = 0; t < R; ++t) o[fpad(base + t * ls)] = x[t];
  }
}

// Transform nlines lines of length d.n (line l at a + l * fline(n), element i
// at fpad(i)) starting at a; b is scratch of the same size. Returns the buffer that holds the result. Must be called
// by all threads of the block; ends with a barrier.
template <bool INV, typename C>
__device__ C* fft_lines(C* a, C* b, int nlines, const FftDesc& d, const C* __restrict__ tw) {
  C* src = a;
  C* dst = b;
  for (int p = 0; p < d.passes; ++p) {
    const C* twp = tw + d.twoff[p];
    switch (d.radix[p]) {
      case 2: fft_pass<2, INV>(src, dst, nlines, d.n, d.ls[p], twp); break;
      case 3: fft_pass<3, INV>(src, dst, nlines, d.n, d.ls[p], twp); break;
      case 4: fft_pass<4, INV>(src, dst, nlines, d.n, d.ls[p], twp); break;
      case 5: fft_pass<5, INV>(src, dst, nlines, d.n, d.ls[p], twp); break;
      case 7: fft_pass<7, INV>(src, dst, nlines, d.n, d.ls[p], twp); break;
      default: fft_pass<8, INV>(src, dst, nlines, d.n, d.ls[p], twp); break;
    }
    __syncthreads();
    C* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

}  // namespace jsd
