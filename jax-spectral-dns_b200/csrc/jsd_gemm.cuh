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
// shared N and strides). Tile shapes and pipeline depth are template
// parameters (DgemmCfg); the plan picks one per call site, by the autotuner
// when asked. A is stored with a zero-padded leading
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

// Tile configuration: BM x BN CTA tile, WM x WN warps (warp tile
// (BM / WM) x (BN / WN), a multiple of 8 x 8), K chunk 16, ST-stage cp.async
// pipeline. B rows are padded to BN + 4 doubles and A rows to 20 doubles, so
// the DMMA fragment loads of a half-warp hit distinct banks.
template <int BM_, int BN_, int WM_, int WN_, int ST_>
struct DgemmCfg {
  static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_, ST = ST_, BK = 16;
  static constexpr int THREADS = 32 * WM * WN;
  static constexpr int TM = BM / WM / 8, TN = BN / WN / 8;
  static constexpr int AS = BK + 4;
  static constexpr int BS = BN + 4;
  static constexpr int A_ELEMS = BM * AS;
  static constexpr int B_ELEMS = BK * BS;
  static constexpr int STAGE = A_ELEMS + B_ELEMS;
  static constexpr size_t BYTES = (size_t)ST * STAGE * sizeof(double);
  static_assert(TM * WM * 8 == BM && TN * WN * 8 == BN, "warp tiles must be multiples of 8 x 8");
};

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS) k_dgemm_t(GemmBatch batch) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, ST = Cfg::ST;
  constexpr int TM = Cfg::TM, TN = Cfg::TN, NT = Cfg::THREADS;
  extern __shared__ __align__(16) double gsm[];

  const GemmEntry& e = batch.e[blockIdx.z];
  const int m0 = blockIdx.y * BM;
  if (m0 >= e.M) return;
  const int n0 = blockIdx.x * BN;
  const int N = batch.N;
  const int lda = batch.lda, ldb = batch.ldb, ldc = batch.ldc;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm = (warp / Cfg::WN) * (BM / Cfg::WM);
  const int wn = (warp % Cfg::WN) * (BN / Cfg::WN);
  // m8 tiles of this warp that hold at least one row of C (warp-uniform)
  int live_tm = (e.M - (m0 + wm) + 7) / 8;
  live_tm = live_tm < 0 ? 0 : (live_tm > TM ? TM : live_tm);

  auto load_chunk = [&](int stage, int k0) {
    double* As = gsm + stage * Cfg::STAGE;
    double* Bs = As + Cfg::A_ELEMS;
    for (int c = tid; c < BM * (BK / 2); c += NT) {
      const int r = c / (BK / 2), cc = (c % (BK / 2)) * 2;
      const int gr = m0 + r;
      const bool ok = gr < e.M;
      const double* src = e.A + (size_t)(ok ? gr : 0) * lda + k0 + cc;
      cp_async16(As + r * Cfg::AS + cc, src, ok ? 16 : 0);
    }
    for (int c = tid; c < BK * (BN / 2); c += NT) {
      const int r = c / (BN / 2), cc = (c % (BN / 2)) * 2;
      const int gk = k0 + r, gn = n0 + cc;
      const bool ok = (gk < e.K) && (gn < N);
      const double* src = e.B + (ok ? ((size_t)gk * ldb + gn) : 0);
      cp_async16(Bs + r * Cfg::BS + cc, src, ok ? 16 : 0);
    }
  };

  double acc[TM][TN][2];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int nchunks = (e.K + BK - 1) / BK;
  // prologue: chunks 0 .. ST-2 in flight (one commit group each, empty groups past the end)
#pragma unroll
  for (int c = 0; c < ST - 1; ++c) {
    if (c < nchunks) load_chunk(c, c * BK);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    // the stage refilled now was last read in iteration c - 1, which every warp has finished
    const int nc = c + ST - 1;
    if (nc < nchunks) load_chunk(nc % ST, nc * BK);
    cp_async_commit();
    const double* As = gsm + (c % ST) * Cfg::STAGE;
    const double* Bs = As + Cfg::A_ELEMS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[TM], bf[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) af[i] = As[(wm + i * 8 + (lane >> 2)) * Cfg::AS + kk + (lane & 3)];
#pragma unroll
      for (int j = 0; j < TN; ++j) bf[j] = Bs[(kk + (lane & 3)) * Cfg::BS + wn + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < TM; ++i)
        if (i < live_tm) {
#pragma unroll
          for (int j = 0; j < TN; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
  }
  cp_async_wait<0>();

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

// Candidate configurations (index = configuration id used by the plan and
// the autotuner).
using DgemmC0 = DgemmCfg<48, 64, 2, 2, 2>;
using DgemmC1 = DgemmCfg<64, 64, 2, 2, 2>;
using DgemmC2 = DgemmCfg<64, 64, 2, 2, 3>;
using DgemmC3 = DgemmCfg<64, 128, 2, 2, 3>;
using DgemmC4 = DgemmCfg<128, 64, 4, 2, 3>;
using DgemmC5 = DgemmCfg<64, 128, 2, 4, 3>;
using DgemmC6 = DgemmCfg<128, 128, 4, 4, 2>;
constexpr int kDgemmConfigs = 7;

// f(Cfg{}) for configuration id `id`
template <typename F>
__host__ bool with_dgemm_cfg(int id, F&& f) {
  switch (id) {
    case 0: f(DgemmC0{}); return true;
    case 1: f(DgemmC1{}); return true;
    case 2: f(DgemmC2{}); return true;
    case 3: f(DgemmC3{}); return true;
    case 4: f(DgemmC4{}); return true;
    case 5: f(DgemmC5{}); return true;
    case 6: f(DgemmC6{}); return true;
    default: return false;
  }
}

// ---------------------------------------------------------------------------
// Split-precision variant for the mixed-precision step: C = A * B with A given
// as two TF32 parts (A = A_hi + A_lo, split on the host from FP64), B read in
// FP64 and split on the fly (b_hi = tf32(b), b_lo = tf32(b - b_hi)), three
// tensor-core products per tile (hi*hi + hi*lo + lo*hi) accumulated in FP32
// (3xTF32), result written in FP64. CTA tile 144 x 64 (one tile covers every
// row of an Ny <= 144 operator), K chunk 16, 6 warps of 48 x 32.
// mma.sync m16n8k8 TF32 fragments (g = lane / 4, t = lane % 4):
//   A a0 (g, t) a1 (g+8, t) a2 (g, t+4) a3 (g+8, t+4); B b0 (t, g) b1 (t+4, g)
//   C c0 (g, 2t) c1 (g, 2t+1) c2 (g+8, 2t) c3 (g+8, 2t+1)
// ---------------------------------------------------------------------------
struct Sgemm3Smem {
  static constexpr int BM = 144, BN = 64, BK = 16;
  static constexpr int AS = BK + 4;  // floats
  static constexpr int BS = BN + 8;  // doubles
  static constexpr int A_BYTES = 2 * BM * AS * 4;
  static constexpr int B_BYTES = BK * BS * 8;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr size_t BYTES = 2 * (size_t)STAGE_BYTES;
  static constexpr int THREADS = 192;
};

struct SplitGemmEntry {
  const float* Ahi;  // M x lda (zero-padded beyond K)
  const float* Alo;
  const double* B;   // K x ldb
  double* C;         // M x ldc
  int M, K;
};

struct SplitGemmBatch {
  SplitGemmEntry e[kGemmMaxBatch];
  int count;
  int N, lda, ldb, ldc;
  int c_f32;  // C holds floats (same element offsets)
};

__device__ __forceinline__ unsigned tf32_bits(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float* d, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(Sgemm3Smem::THREADS) k_sgemm3(SplitGemmBatch batch) {
  using S = Sgemm3Smem;
  constexpr int BN = S::BN, BK = S::BK, BM = S::BM;
  constexpr int TM = 3, TN = 4;
  extern __shared__ __align__(16) unsigned char ssm[];

  const SplitGemmEntry& e = batch.e[blockIdx.z];
  const int n0 = blockIdx.x * BN;
  const int N = batch.N;
  const int lda = batch.lda, ldb = batch.ldb, ldc = batch.ldc;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 1) * 48;
  const int wn = (warp & 1) * 32;

  auto load_chunk = [&](int stage, int k0) {
    float* Ah = reinterpret_cast<float*>(ssm + stage * S::STAGE_BYTES);
    float* Al = Ah + BM * S::AS;
    double* Bs = reinterpret_cast<double*>(ssm + stage * S::STAGE_BYTES + S::A_BYTES);
    // A parts: BM rows x 16 floats = 4 copies of 16 bytes per row and part
    for (int c = tid; c < 2 * BM * (BK / 4); c += S::THREADS) {
      const int part = c / (BM * (BK / 4));
      const int cc_ = c - part * BM * (BK / 4);
      const int r = cc_ / (BK / 4), cc = (cc_ % (BK / 4)) * 4;
      const bool ok = r < e.M;
      const float* base = part ? e.Alo : e.Ahi;
      const float* src = base + (size_t)(ok ? r : 0) * lda + k0 + cc;
      cp_async16((part ? Al : Ah) + r * S::AS + cc, src, ok ? 16 : 0);
    }
    for (int c = tid; c < BK * (BN / 2); c += S::THREADS) {
      const int r = c / (BN / 2), cc = (c % (BN / 2)) * 2;
      const int gk = k0 + r, gn = n0 + cc;
      const bool ok = (gk < e.K) && (gn < N);
      const double* src = e.B + (ok ? ((size_t)gk * ldb + gn) : 0);
      cp_async16(Bs + r * S::BS + cc, src, ok ? 16 : 0);
    }
    cp_async_commit();
  };

  float acc[TM][TN][4];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

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
    const float* Ah = reinterpret_cast<const float*>(ssm + (c & 1) * S::STAGE_BYTES);
    const float* Al = Ah + BM * S::AS;
    const double* Bs = reinterpret_cast<const double*>(ssm + (c & 1) * S::STAGE_BYTES + S::A_BYTES);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      unsigned bh[TN][2], bl[TN][2];
#pragma unroll
      for (int j = 0; j < TN; ++j)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const float x = (float)Bs[(kk + t + 4 * q) * S::BS + wn + j * 8 + g];
          const unsigned h = tf32_bits(x);
          bh[j][q] = h;
          bl[j][q] = tf32_bits(x - __uint_as_float(h));
        }
#pragma unroll
      for (int i = 0; i < TM; ++i) {
        unsigned ah[4], al[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int row = wm + i * 16 + g + 8 * (q & 1);
          const int col = kk + t + 4 * (q >> 1);
          ah[q] = __float_as_uint(Ah[row * S::AS + col]);
          al[q] = __float_as_uint(Al[row * S::AS + col]);
        }
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          mma_tf32(acc[i][j], al, bh[j]);
          mma_tf32(acc[i][j], ah, bl[j]);
          mma_tf32(acc[i][j], ah, bh[j]);
        }
      }
    }
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < TM; ++i) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = wm + i * 16 + g + 8 * h;
      if (r >= e.M) continue;
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int col = n0 + wn + j * 8 + 2 * t;
        if (col < N) {
          if (batch.c_f32)
            *reinterpret_cast<float2*>(reinterpret_cast<float*>(e.C) + (size_t)r * ldc + col) =
                make_float2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
          else
            *reinterpret_cast<double2*>(e.C + (size_t)r * ldc + col) =
                make_double2((double)acc[i][j][2 * h], (double)acc[i][j][2 * h + 1]);
        }
      }
    }
  }
}

}  // namespace jsd
