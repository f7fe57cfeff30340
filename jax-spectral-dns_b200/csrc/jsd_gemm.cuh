// FP64 y-contractions on the FP64 tensor cores (DMMA, mma.sync m8n8k4.f64).
//
// Every y-direction operator of the step (Chebyshev derivative D, the D^2
// eigenbasis transforms and their combinations) is a real Ny-sized matrix
// applied to all (kx, kz) columns at once. With spectral fields stored plane
// by plane, a field is a row-major K x N matrix (N = 2 mx mz doubles: real and
// imaginary parts are independent columns because the operators are real), so
// each application is C (M x N) = alpha * A (M x K) * B (K x N).
//
// One launch runs a small batch of such products (different A, B, C, M, K;
// shared N and strides). CTA tile BM x 64, K chunk 16, two-stage cp.async
// pipeline, 4 warps of (BM/2) x 32. A is stored with a zero-padded leading
// dimension (multiple of 16); rows of B beyond K and columns beyond N are
// zero-filled by the copy, so no out-of-range element is read.
#pragma once

#include "jsd_common.cuh"

namespace jsd {

constexpr int kGemmMaxBatch = 8;

struct GemmEntry {
  const double* A;  // M x lda, zero-padded beyond K
  const double* B;  // K x ldb (first row = first row used)
  double* C;        // M x ldc
  int M, K;
  double alpha;
};

struct GemmBatch {
  GemmEntry e[kGemmMaxBatch];
  int count;
  int N, lda, ldb, ldc;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int BM>
struct GemmSmem {
  static constexpr int BN = 64, BK = 16;
  static constexpr int AS = BK + 4;   // A row stride (doubles): conflict-free fragment loads
  static constexpr int BS = BN + 8;   // B row stride (doubles)
  static constexpr int A_ELEMS = BM * AS;
  static constexpr int B_ELEMS = BK * BS;
  static constexpr int STAGE = A_ELEMS + B_ELEMS;
  static constexpr size_t BYTES = 2 * STAGE * sizeof(double);
};

template <int BM>
__global__ void __launch_bounds__(128) k_dgemm(GemmBatch batch) {
  using S = GemmSmem<BM>;
  constexpr int BN = S::BN, BK = S::BK;
  constexpr int TM = BM / 16;  // m8 tiles per warp (warp tile BM/2 rows)
  constexpr int TN = 4;        // n8 tiles per warp (warp tile 32 cols)
  extern __shared__ __align__(16) double gsm[];

  const GemmEntry& e = batch.e[blockIdx.z];
  const int m0 = blockIdx.y * BM;
  if (m0 >= e.M) return;
  const int n0 = blockIdx.x * BN;
  const int N = batch.N;
  const int lda = batch.lda, ldb = batch.ldb, ldc = batch.ldc;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm = (warp >> 1) * (BM / 2);
  const int wn = (warp & 1) * 32;

  auto load_chunk = [&](int stage, int k0) {
    double* As = gsm + stage * S::STAGE;
    double* Bs = As + S::A_ELEMS;
    // A: BM rows x 16 doubles = BM * 8 copies of 16 bytes
    for (int c = tid; c < BM * (BK / 2); c += 128) {
      const int r = c / (BK / 2), cc = (c % (BK / 2)) * 2;
      const int gr = m0 + r;
      const bool ok = gr < e.M;
      const double* src = e.A + (size_t)(ok ? gr : 0) * lda + k0 + cc;
      cp_async16(As + r * S::AS + cc, src, ok ? 16 : 0);
    }
    // B: 16 rows x 64 doubles = 512 copies
    for (int c = tid; c < BK * (BN / 2); c += 128) {
      const int r = c / (BN / 2), cc = (c % (BN / 2)) * 2;
      const int gk = k0 + r, gn = n0 + cc;
      const bool ok = (gk < e.K) && (gn < N);
      const double* src = e.B + (ok ? ((size_t)gk * ldb + gn) : 0);
      cp_async16(Bs + r * S::BS + cc, src, ok ? 16 : 0);
    }
    cp_async_commit();
  };

  double acc[TM][TN][2];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int nchunks = (e.K + BK - 1) / BK;
  load_chunk(0, 0);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      load_chunk((c + 1) & 1, (c + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* As = gsm + (c & 1) * S::STAGE;
    const double* Bs = As + S::A_ELEMS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[TM], bf[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) af[i] = As[(wm + i * 8 + (lane >> 2)) * S::AS + kk + (lane & 3)];
#pragma unroll
      for (int j = 0; j < TN; ++j) bf[j] = Bs[(kk + (lane & 3)) * S::BS + wn + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }

  const double alpha = e.alpha;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int r = m0 + wm + i * 8 + (lane >> 2);
    if (r >= e.M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int col = n0 + wn + j * 8 + 2 * (lane & 3);
      if (col < N) {
        *reinterpret_cast<double2*>(e.C + (size_t)r * ldc + col) =
            make_double2(alpha * acc[i][j][0], alpha * acc[i][j][1]);
      }
    }
  }
}

}  // namespace jsd
