// Split-TF32 y-derivatives on the 5th-generation tensor cores (tcgen05).
//
// C (M x N, FP64) = D (M x K) * B (K x N, FP64) for M <= 128 rows of the
// Chebyshev matrix, as three TF32 products D_hi B_hi + D_hi B_lo + D_lo B_hi
// accumulated in FP32 in tensor memory (the same 3xTF32 scheme as k_sgemm3).
//
// One persistent CTA of 4 warps per SM:
//   * D_hi and D_lo (pre-arranged on the host in the canonical K-major
//     core-matrix layout, 128 rows x 136 K) arrive once by bulk copy
//     (cp.async.bulk, completion on an mbarrier) and stay in shared memory;
//   * per 64-column tile, the warps split the FP64 B tile into TF32 hi / lo
//     core matrices in shared memory, one elected thread issues
//     3 x ceil(K/8) tcgen05.mma.kind::tf32 (M = 128, N = 64, K = 8) into a
//     128 x 64 FP32 accumulator in TMEM and commits to an mbarrier;
//   * the warps read the accumulator back with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = rows), widen to FP64 and store through a padded
//     shared-memory stage so the global writes are row-contiguous.
// Every wait on an mbarrier has an iteration limit; on expiry the kernel sets
// the error flag, skips the remaining tiles, frees its TMEM and returns.
//
// Canonical K-major layout without swizzle (units of 16 bytes = 4 TF32): a core
// matrix is 8 rows x 16 bytes stored contiguously; core matrix (row group g,
// K chunk c) of an R-row operand sits at byte (c * R / 8 + g) * 128. In the
// shared-memory descriptor the stride byte offset (between row groups) is 128
// and the leading byte offset (between the two K chunks of one MMA) is R * 16.
#pragma once

#include <cstdint>
#include <vector>

#include "jsd_common.cuh"
#include "jsd_gemm.cuh"

namespace jsd {

constexpr int kTcM = 128;                      // accumulator rows (TMEM lanes)
constexpr int kTcN = 64;                       // columns per tile (TMEM columns)
constexpr int kTcKp = 136;                     // padded K (17 MMA steps of 8)
constexpr int kTcASize = kTcM * kTcKp * 4;     // bytes of one A part (69632)
constexpr int kTcBSize = kTcN * kTcKp * 4;     // bytes of one B part (34816)
constexpr int kTcStageLd = kTcN + 1;           // padded row of the FP64 output stage
constexpr int kTcBatch = 17;                   // tile loads in flight per thread during the conversion
constexpr size_t kTcSmem = 2 * (size_t)kTcASize + 2 * (size_t)kTcBSize + 64;
static_assert((size_t)kTcM * kTcStageLd * 8 <= 2 * (size_t)kTcBSize, "output stage must fit in the B tiles");

struct Tc05Batch {
  const double* B[kGemmMaxBatch];
  double* C[kGemmMaxBatch];
  int count;
  int M, N, K, ldb, ldc;
};

// byte offset of element (row r, k) of an R-row operand in the core-matrix layout
__host__ __device__ __forceinline__ int tc05_offset(int R, int r, int k) {
  return ((k >> 2) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ uint32_t tc_smem(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t tc05_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version 1; base offset 0, no swizzle
  return d;
}

// F32 accumulator, TF32 A and B, both K-major, N = 64 (>> 3), M = 128 (>> 4)
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                              ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(acc), "r"(0u));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

// true when the phase of `parity` completed within the iteration limit
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ float tf32_round_dev(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}
#endif

// B[i] / C[i] by selects (a runtime index into the kernel parameter would copy
// the parameter arrays to local memory)
__device__ __forceinline__ void tc05_entry(const Tc05Batch& b, int e, const double*& B, double*& C) {
  B = b.B[0];
  C = b.C[0];
#pragma unroll
  for (int i = 1; i < kGemmMaxBatch; ++i)
    if (e == i) {
      B = b.B[i];
      C = b.C[i];
    }
}

__global__ void __launch_bounds__(128, 1) k_tc05_dfield(const float* __restrict__ a_hi, const float* __restrict__ a_lo,
                                                       Tc05Batch b, int* __restrict__ err) {
#if defined(__CUDA_ARCH__)
  extern __shared__ __align__(1024) unsigned char tsm[];
  float* sAh = reinterpret_cast<float*>(tsm);
  float* sAl = sAh + kTcASize / 4;
  float* sBh = sAl + kTcASize / 4;
  float* sBl = sBh + kTcBSize / 4;
  double* stage = reinterpret_cast<double*>(sBh);  // output stage reuses the B tiles after the MMAs
  uint64_t* bars = reinterpret_cast<uint64_t*>(tsm + 2 * kTcASize + 2 * kTcBSize);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar_a = tc_smem(&bars[0]), bar_m = tc_smem(&bars[1]);
  if (tid == 0) {
    mbar_init(bar_a, 1);
    mbar_init(bar_m, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc_smem(tslot)),
                 "r"((uint32_t)kTcN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar_a),
                 "r"((uint32_t)(2 * kTcASize))
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     tc_smem(sAh)),
                 "l"(a_hi), "r"((uint32_t)kTcASize), "r"(bar_a)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     tc_smem(sAl)),
                 "l"(a_lo), "r"((uint32_t)kTcASize), "r"(bar_a)
                 : "memory");
  }
  int ok = __syncthreads_and(mbar_wait(bar_a, 0) ? 1 : 0);
  const int ksteps = (b.K + 7) / 8;  // <= kTcKp / 8
  const int tiles_n = (b.N + kTcN - 1) / kTcN;
  const int ntiles = tiles_n * b.count;
  const uint32_t lbo_a = kTcM * 16, lbo_b = kTcN * 16;
  uint32_t phase = 0;
  for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
    const int e = tile / tiles_n;
    const int n0 = (tile - e * tiles_n) * kTcN;
    const double* B;
    double* C;
    tc05_entry(b, e, B, C);
    // B tile -> TF32 hi / lo core matrices. A warp fills one core matrix
    // (8 columns x 4 K, lane = (column, K) pair) per pass; each thread first
    // issues the loads of kTcBatch passes, then converts and stores them, so
    // that many loads are in flight.
    const int ncm = (kTcN / 8) * (2 * ksteps);
    for (int cm0 = warp; cm0 < ncm; cm0 += 4 * kTcBatch) {
      double v[kTcBatch];
#pragma unroll
      for (int q = 0; q < kTcBatch; ++q) {
        const int cm = cm0 + 4 * q;
        const int g = cm % (kTcN / 8), c = cm / (kTcN / 8);
        const int n = g * 8 + (lane >> 2), k = c * 4 + (lane & 3);
        v[q] = (cm < ncm && k < b.K && n0 + n < b.N) ? B[(size_t)k * b.ldb + n0 + n] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < kTcBatch; ++q) {
        const int cm = cm0 + 4 * q;
        if (cm >= ncm) break;
        const int g = cm % (kTcN / 8), c = cm / (kTcN / 8);
        const int n = g * 8 + (lane >> 2), k = c * 4 + (lane & 3);
        const float h = tf32_round_dev((float)v[q]);
        const float l = tf32_round_dev((float)(v[q] - (double)h));
        const int off = tc05_offset(kTcN, n, k) >> 2;
        sBh[off] = h;
        sBl[off] = l;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      // K step s moves the start-address field (address / 16) by a constant
      const uint64_t dah = tc05_desc(tc_smem(sAh), lbo_a, 128), dal = tc05_desc(tc_smem(sAl), lbo_a, 128);
      const uint64_t dbh = tc05_desc(tc_smem(sBh), lbo_b, 128), dbl = tc05_desc(tc_smem(sBl), lbo_b, 128);
#pragma unroll
      for (int s = 0; s < kTcKp / 8; ++s) {
        if (s >= ksteps) break;
        const uint64_t oa = (2u * s * lbo_a) >> 4, ob = (2u * s * lbo_b) >> 4;
        tc_mma(tmem, dah + oa, dbh + ob, s > 0 ? 1u : 0u);
        tc_mma(tmem, dah + oa, dbl + ob, 1u);
        tc_mma(tmem, dal + oa, dbh + ob, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_m)
                   : "memory");
    }
    ok = __syncthreads_and(mbar_wait(bar_m, phase) ? 1 : 0);
    phase ^= 1u;
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // accumulator rows 32 warp + lane -> FP64 stage
    const int r = 32 * warp + lane;
#pragma unroll
    for (int q = 0; q < kTcN / 16; ++q) {
      float v[16];
      tc_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(16 * q), v);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) stage[r * kTcStageLd + 16 * q + j] = (double)v[j];
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    for (int i = tid; i < kTcM * kTcN; i += blockDim.x) {
      const int rr = i / kTcN, jj = i - (i / kTcN) * kTcN;
      if (rr < b.M && n0 + jj < b.N) C[(size_t)rr * b.ldc + n0 + jj] = stage[rr * kTcStageLd + jj];
    }
    __syncthreads();
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)kTcN));
  }
#endif
}

// Host: rows 0..M-1 of D (row-major, ld = ldd) split into TF32 hi / lo in the
// core-matrix layout of a 128-row operand (rows >= M and K >= k zero).
inline void tc05_pack_a(const double* D, int M, int K, int ldd, float (*tf32)(float), std::vector<float>& hi,
                        std::vector<float>& lo) {
  hi.assign(kTcASize / 4, 0.f);
  lo.assign(kTcASize / 4, 0.f);
  for (int r = 0; r < M && r < kTcM; ++r)
    for (int k = 0; k < K && k < kTcKp; ++k) {
      const double x = D[(size_t)r * ldd + k];
      const float h = tf32((float)x);
      const int off = tc05_offset(kTcM, r, k) >> 2;
      hi[off] = h;
      lo[off] = tf32((float)(x - (double)h));
    }
}

}  // namespace jsd
