// tcgen05 building blocks (shared-memory descriptors, mbarriers with bounded
// waits, bulk and TMA copies, tensor-memory loads) and the split-TF32
// y-derivative kernel on the 5th-generation tensor cores.
//
// k_tc05_dfield: C (M x N, FP64) = D (M x K) * B (K x N, FP64) for the
// Chebyshev derivative matrix D (M = K = Ny <= 129), as three TF32 products
// D_hi B_hi + D_lo B_hi + D_hi B_lo with FP32 accumulation in tensor memory
// (the same 3xTF32 scheme as k_sgemm3). One persistent CTA of 27 warps per SM,
// each CTA a contiguous range of 32-column tiles:
//   * warp 26 (producer): one 2-D TMA load (cp.async.bulk.tensor, mbarrier
//     completion) of the tile's 136 x 32 FP64 block of B into a staging buffer
//     (rows past K and columns past N arrive as zeros);
//   * warps 0-16 (converters, warp w = rows 8w..8w+7, lane = column): split the
//     staged values into TF32 hi and lo and store them as one 64-row K-major
//     operand (hi rows 0-31, lo rows 32-63); for Ny = 129 they also form the
//     FP64 dot products of D's last row (y = -1) with their rows;
//   * warp 25 (issuer): keeps D_hi / D_lo resident (bulk copy once), issues per
//     K step of 8 two tcgen05.mma.kind::tf32 (M = 128): D_hi x [B_hi; B_lo]
//     (N = 64: hi*hi into columns 0-31, hi*lo into 32-63) and D_lo x B_hi
//     (N = 32, into columns 0-31), into one of two 64-column accumulator sets;
//   * warps 17-24 (epilogue, TMEM lane quadrant = warp % 4, half of the
//     columns each): read both accumulators (tcgen05.ld), add them in FP64 and
//     store; the last row (Ny = 129) from the converters' partial dots.
// Every mbarrier wait has an iteration limit (a kernel argument); on expiry the
// kernel raises the error flag, every role stops at its next tile, the issuer
// waits (bounded) for its operand copy and its last MMAs, the producer for its
// last staged load, and the CTA frees its TMEM and returns.
//
// Canonical K-major layout without swizzle (units of 16 bytes = 4 TF32): a core
// matrix is 8 rows x 16 bytes stored contiguously; core matrix (row group g,
// K chunk c) of an R-row operand sits at byte (c * R / 8 + g) * 128. In the
// shared-memory descriptor the stride byte offset (between row groups) is 128
// and the leading byte offset (between the two K chunks of one MMA) is R * 16.
#pragma once

#include <cuda.h>  // CUtensorMap

#include <cstdint>
#include <vector>

#include "jsd_common.cuh"
#include "jsd_gemm.cuh"

namespace jsd {

// Polls of an mbarrier before a pipeline wait gives up (the plan's default;
// jsd_set_wait_limit changes it), and before a CTA that gave up stops waiting
// for its own copies and MMAs in flight before it tears down.
constexpr int kWaitPolls = 1 << 22;
constexpr int kDrainPolls = 1 << 22;

constexpr int kTcM = 128;                      // accumulator rows (TMEM lanes)
constexpr int kTcKp = 136;                     // padded K (17 MMA steps of 8)
constexpr int kTcN = 32;                       // columns per tile
constexpr int kTcASize = kTcM * kTcKp * 4;     // bytes of one A part (69632)
constexpr int kTcBRows = 2 * kTcN;             // stacked B operand rows (hi, lo)
constexpr int kTcBSize = kTcBRows * kTcKp * 4;  // 34816
constexpr int kTcStageBytes = kTcKp * kTcN * 8;  // 34816
constexpr int kTcConvWarps = kTcKp / 8, kTcEpiWarps = 8;
constexpr int kTcIssuerWarp = kTcConvWarps + kTcEpiWarps, kTcProducerWarp = kTcIssuerWarp + 1;
constexpr int kTcThreads = 32 * (kTcProducerWarp + 1);  // 864
constexpr int kTcSideDoubles = kTcConvWarps * kTcN;      // partial dots of the last row
constexpr int kTcTmemCols = 2 * 2 * kTcN;                // two sets of (hi*hi + lo*hi, hi*lo)
constexpr size_t kTcSmem =
    2 * (size_t)kTcASize + kTcBSize + kTcStageBytes + 2 * sizeof(double) * kTcSideDoubles + 128;

// map: 2-D tensor map of B[i] (inner N doubles, outer K rows, row stride
// ldb), box 32 x 136
struct Tc05Batch {
  CUtensorMap map[kGemmMaxBatch];
  double* C[kGemmMaxBatch];
  const double* xrow;  // M = 129: row 128 of D (K values), else null
  int count;
  int M, N, K, ldb, ldc;
};

// byte offset of element (row r, k) of an R-row TF32 operand in the core-matrix layout
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

// F32 accumulator, TF32 A and B, both K-major, M = 128, N as given
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

// true when the phase of `parity` completed within `limit` polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
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

// TMA store of a 2-D box from shared memory (x: innermost, a multiple of 16
// bytes, both coordinates >= 0; elements outside the tensor are not written),
// tracked in the issuing thread's bulk async-group
__device__ __forceinline__ void tc_tma_store_2d(const CUtensorMap* map, int x, int y, const void* src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(map), "r"(x),
               "r"(y), "r"(tc_smem(src))
               : "memory");
}
__device__ __forceinline__ void tc_bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the shared-memory sources of this thread's bulk stores may be overwritten
__device__ __forceinline__ void tc_bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// this thread's bulk stores are complete
__device__ __forceinline__ void tc_bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void tc_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tc_bulk_g2s(void* dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   tc_smem(dst)),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// 2-D TMA load of the box at (x, y) (x: innermost, a multiple of 16 bytes)
__device__ __forceinline__ void tc_tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          tc_smem(dst)),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ float tf32_round_dev(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
#endif

__global__ void __launch_bounds__(kTcThreads, 1) k_tc05_dfield(const float* __restrict__ a_hi,
                                                               const float* __restrict__ a_lo,
                                                               const __grid_constant__ Tc05Batch b,
                                                               int* __restrict__ err, int spin) {
#if defined(__CUDA_ARCH__)
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* sAh = tsm;
  unsigned char* sAl = tsm + kTcASize;
  unsigned char* sB = tsm + 2 * kTcASize;                       // stacked hi / lo operand
  double* stage = reinterpret_cast<double*>(sB + kTcBSize);      // staged FP64 tile, row k at 32 k
  double* side = stage + kTcKp * kTcN;                          // two tile buffers of partial dots
  uint64_t* bars = reinterpret_cast<uint64_t*>(side + 2 * kTcSideDoubles);
  // bars: 0,1 full (B operand + partial dots of tile parity); 2,3 mma done;
  // 4,5 epilogue done; 6 A loaded; 7 staged tile ready; 8 staging released
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 9);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto bar = [&](int i) { return tc_smem(&bars[i]); };
  if (tid == 0) {
    mbar_init(bar(0), 32 * kTcConvWarps);
    mbar_init(bar(1), 32 * kTcConvWarps);
    mbar_init(bar(2), 1);
    mbar_init(bar(3), 1);
    mbar_init(bar(4), 32 * kTcEpiWarps);
    mbar_init(bar(5), 32 * kTcEpiWarps);
    mbar_init(bar(6), 1);
    mbar_init(bar(7), 1);
    mbar_init(bar(8), 32 * kTcConvWarps);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc_smem(tslot)),
                 "r"((uint32_t)kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  const int tiles_n = (b.N + kTcN - 1) / kTcN;
  const long long total = (long long)tiles_n * b.count;
  const int t_begin = (int)(total * blockIdx.x / gridDim.x);
  const int t_end = (int)(total * (blockIdx.x + 1) / gridDim.x);
  const int nt = t_end - t_begin;
  const int ksteps = (b.K + 7) / 8;  // <= kTcKp / 8
  auto fail_now = [&]() {
    *abort_flag = 1;
    atomicOr(err, kErrWaitExpired);
  };

  if (warp < kTcConvWarps) {
    // ---------------------------------------------------------------- converters
    const int n = lane, k0 = 8 * warp;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kTcN;
      const bool cv = n0 + n < b.N;
      bool ok = mbar_wait(bar(7), i & 1, spin);
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        break;
      }
      double x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = cv ? stage[(k0 + j) * kTcN + n] : 0.0;  // rows >= K arrive as zeros
      tc_arrive(bar(8));  // staging may be refilled
      double dot = 0.0;
      if (b.M > kTcM) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (k0 + j < b.K) dot = fma(__ldg(b.xrow + k0 + j), x[j], dot);
      }
      uint32_t hi[8], lo[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float h = tf32_round_dev((float)x[j]);
        hi[j] = __float_as_uint(h);
        lo[j] = __float_as_uint(tf32_round_dev((float)(x[j] - (double)h)));
      }
      // the B operand is free once the previous tile's MMAs completed; the
      // partial dots once the epilogue of the tile two back is done
      ok = (i < 1 || mbar_wait(bar(2 + ((i - 1) & 1)), ((i - 1) >> 1) & 1, spin)) &&
           (i < 2 || mbar_wait(bar(4 + buf), ((i - 2) >> 1) & 1, spin));
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        break;
      }
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        *reinterpret_cast<uint4*>(sB + tc05_offset(kTcBRows, n, k0 + 4 * c)) =
            make_uint4(hi[4 * c], hi[4 * c + 1], hi[4 * c + 2], hi[4 * c + 3]);
        *reinterpret_cast<uint4*>(sB + tc05_offset(kTcBRows, kTcN + n, k0 + 4 * c)) =
            make_uint4(lo[4 * c], lo[4 * c + 1], lo[4 * c + 2], lo[4 * c + 3]);
      }
      side[buf * kTcSideDoubles + warp * kTcN + n] = dot;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      tc_arrive(bar(buf));
    }
  } else if (warp < kTcConvWarps + kTcEpiWarps) {
    // ----------------------------------------------------------------- epilogue
    const int ew = warp - kTcConvWarps, quad = warp & 3, half = ew >> 2;
    const int row = 32 * quad + lane, c0 = 16 * half;
    const int mt = b.M < kTcM ? b.M : kTcM;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      const bool ok = mbar_wait(bar(2 + buf), (i >> 1) & 1, spin) && mbar_wait(bar(buf), (i >> 1) & 1, spin);
      if (!__all_sync(0xffffffffu, ok)) {  // tcgen05.ld below needs the whole warp
        fail_now();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kTcN;
      double* C = b.C[0];
#pragma unroll
      for (int q = 1; q < kGemmMaxBatch; ++q)
        if (e == q) C = b.C[q];
      const uint32_t tbase = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(buf * 2 * kTcN + c0);
      uint32_t s0[16], s1[16];
      tc_ld16(tbase, s0);           // hi*hi + lo*hi
      tc_ld16(tbase + kTcN, s1);    // hi*lo
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      if (row < mt) {
        double* out = C + (size_t)row * b.ldc + n0 + c0;
        if (n0 + c0 + 16 <= b.N) {
#pragma unroll
          for (int j = 0; j < 16; j += 2)
            *reinterpret_cast<double2*>(out + j) =
                make_double2((double)__uint_as_float(s0[j]) + (double)__uint_as_float(s1[j]),
                             (double)__uint_as_float(s0[j + 1]) + (double)__uint_as_float(s1[j + 1]));
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (n0 + c0 + j < b.N) out[j] = (double)__uint_as_float(s0[j]) + (double)__uint_as_float(s1[j]);
        }
      }
      if (b.M > kTcM && ew == 0 && n0 + lane < b.N) {
        const double* sd = side + buf * kTcSideDoubles;
        double x = sd[lane];
#pragma unroll
        for (int w = 1; w < kTcConvWarps; ++w) x += sd[w * kTcN + lane];
        C[(size_t)kTcM * b.ldc + n0 + lane] = x;
      }
      tc_arrive(bar(4 + buf));
    }
  } else if (warp == kTcIssuerWarp) {
    // ------------------------------------------------------------------- issuer
    if (lane == 0) {
      int issued = 0;
      tc_expect_tx(bar(6), (uint32_t)(2 * kTcASize));
      tc_bulk_g2s(sAh, a_hi, (uint32_t)kTcASize, bar(6));
      tc_bulk_g2s(sAl, a_lo, (uint32_t)kTcASize, bar(6));
      if (!mbar_wait(bar(6), 0, spin)) {
        fail_now();
        // the operand copy may still be writing shared memory: let it land
        if (!mbar_wait(bar(6), 0, kDrainPolls)) atomicOr(err, kErrWaitExpired);
      }
      constexpr uint32_t lbo_a = kTcM * 16, lbo_b = kTcBRows * 16;
      const uint64_t dah = tc05_desc(tc_smem(sAh), lbo_a, 128), dal = tc05_desc(tc_smem(sAl), lbo_a, 128);
      const uint64_t db = tc05_desc(tc_smem(sB), lbo_b, 128);
      for (int i = 0; i < nt && !*abort_flag; ++i) {
        const int buf = i & 1;
        if (!mbar_wait(bar(buf), (i >> 1) & 1, spin)) {
          fail_now();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(buf * 2 * kTcN);
        // K step s moves the start-address field (address / 16) by a constant
#pragma unroll
        for (int s = 0; s < kTcKp / 8; ++s) {
          if (s >= ksteps) break;
          const uint64_t oa = (2u * s * lbo_a) >> 4, ob = (2u * s * lbo_b) >> 4;
          tc_mma_tf32(acc, dah + oa, db + ob, tc_idesc_tf32(2 * kTcN), s > 0 ? 1u : 0u);  // hi x [hi; lo]
          tc_mma_tf32(acc, dal + oa, db + ob, tc_idesc_tf32(kTcN), 1u);                 // lo x hi
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         bar(2 + buf))
                     : "memory");
        issued = i + 1;
      }
      // no MMA may still run when the CTA frees its tensor memory
      if (issued > 0 && !mbar_wait(bar(2 + ((issued - 1) & 1)), ((issued - 1) >> 1) & 1, kDrainPolls)) fail_now();
    }
  } else {
    // ----------------------------------------------------------------- producer
    int loads = 0;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kTcN;
      const bool ok = i < 1 || mbar_wait(bar(8), (i - 1) & 1, spin);
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        break;
      }
      if (lane == 0) {
        tc_expect_tx(bar(7), (uint32_t)kTcStageBytes);
        tc_tma_load_2d(stage, &b.map[e], n0, 0, bar(7));
      }
      ++loads;
    }
    // one staged load at most is in flight (the next is issued only after the
    // converters read the previous one): wait for it before the CTA's shared
    // memory is released (returns at once when every load was consumed)
    if (lane == 0 && loads > 0 && !mbar_wait(bar(7), (loads - 1) & 1, kDrainPolls)) atomicOr(err, kErrWaitExpired);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)kTcTmemCols));
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
