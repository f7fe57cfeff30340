// Shared device helpers for the velocity-vorticity channel step.
//
// Spectral fields are stored plane by plane: element (y, ix, iz) of a field
// lives at ((y * mx + ix) * mz + iz) as an interleaved complex double (re, im)
// (for a batch of runs, y is the plane index y_cheb * nb + run).
// A vector field is three such fields back to back. Wavenumber indices follow
// the FFT order of the reference ([0..K, -K..-1]); y index 0 is y = +1.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace jsd {

// bits of a plan's device error flag
constexpr int kErrWaitExpired = 1;  // a pipeline wait of a tcgen05 kernel gave up (its results are invalid)
constexpr int kErrNonFinite = 2;    // a stage produced a NaN or an infinity

struct Geo {
  int mx, ny, mz;    // Fourier modes in x and z (odd), Chebyshev points in y
  int kx_max, kz_max;  // K = m / 2
  int px, pz;        // FFT lengths used on the device (>= 3K + 1)
  int nk;            // mx * mz
  double ax, az;     // wavenumber units 2 pi / Lx, 2 pi / Lz
  double c_inv;      // s / sqrt(Px_ref Pz_ref): coefficient -> physical value
  double c_fwd;      // sqrt(Px_ref Pz_ref) / (s px pz): unnormalised DFT -> coefficient
  int nb;            // runs stepped together (1: a single run). A batch stores each field
                     // as [y][run][kx][kz]: plane p = y * nb + run, and a Chebyshev row
                     // holds nb * nk modes. Kernels that only see planes get ny = planes.
};

// complex helpers for double2 (FP64 path) and float2 (FP32 transforms of the
// mixed-precision path)
template <typename T> struct real_of;
template <> struct real_of<double2> { using type = double; };
template <> struct real_of<float2> { using type = float; };

__host__ __device__ __forceinline__ double2 mkc(double x, double y, double2*) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 mkc(float x, float y, float2*) { return make_float2(x, y); }
template <typename C>
__host__ __device__ __forceinline__ C cmake(typename real_of<C>::type x, typename real_of<C>::type y) {
  return mkc(x, y, (C*)nullptr);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 cmul_ik(float2 a, float k) { return make_float2(-k * a.y, k * a.x); }
template <typename C> __host__ __device__ __forceinline__ C to_c(double2 a) { return cmake<C>(a.x, a.y); }
template <typename C> __host__ __device__ __forceinline__ C to_c(float2 a) { return cmake<C>(a.x, a.y); }

__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// i * k * a
__host__ __device__ __forceinline__ double2 cmul_ik(double2 a, double k) { return make_double2(-k * a.y, k * a.x); }

// signed mode index of position i in an FFT-ordered array of m = 2K + 1 entries
__host__ __device__ __forceinline__ int signed_mode(int i, int m) { return i <= m / 2 ? i : i - m; }
// position of signed mode k
__host__ __device__ __forceinline__ int mode_pos(int k, int m) { return k >= 0 ? k : k + m; }

__host__ __device__ __forceinline__ double kx_of(const Geo& g, int ix) { return signed_mode(ix, g.mx) * g.ax; }
__host__ __device__ __forceinline__ double kz_of(const Geo& g, int iz) { return signed_mode(iz, g.mz) * g.az; }

__host__ __device__ __forceinline__ size_t sidx(const Geo& g, int y, int ix, int iz) {
  return ((size_t)y * g.mx + ix) * g.mz + iz;
}

// `bytes` (a multiple of 16) from a 16-byte aligned global address into L2
__device__ __forceinline__ void l2_prefetch(const void* p, unsigned bytes) {
#if defined(__CUDA_ARCH__)
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
#endif
}

// Hermitian part of X at the signed mode (kx, kz): (X(k) + conj X(-k)) / 2.
__host__ __device__ __forceinline__ double2 sym_at(const Geo& g, const double2* __restrict__ f, int y, int kx, int kz) {
  double2 a = f[sidx(g, y, mode_pos(kx, g.mx), mode_pos(kz, g.mz))];
  double2 b = f[sidx(g, y, mode_pos(-kx, g.mx), mode_pos(-kz, g.mz))];
  return make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
}

// The reference's forward-transform truncation keeps the true coefficients for
// |k| <= K except that, axis by axis (x first, then z), the -K slot receives
// the conjugate of the +K slot of the array as it stands at that point. For an
// output slot (ix, iz) this reduces to: read the true coefficient at
// (kx', kz') where a -K slot is replaced by +K, and conjugate once per replaced
// axis. This helper returns (kx', kz') and the parity of conjugations.
__host__ __device__ __forceinline__ void truncation_source(const Geo& g, int ix, int iz, int& kx, int& kz, bool& conj) {
  const bool sx = (ix == g.kx_max + 1);
  const bool sz = (iz == g.kz_max + 1);
  kx = sx ? g.kx_max : signed_mode(ix, g.mx);
  kz = sz ? g.kz_max : signed_mode(iz, g.mz);
  conj = (sx != sz);
}

}  // namespace jsd
