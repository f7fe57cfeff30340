// tcgen05 building blocks (shared-memory descriptors, mbarriers with bounded
// waits, bulk and TMA copies, tensor-memory loads) and the split-TF32 product
// kernel on the 5th-generation tensor cores.
//
// k_tc05_split: C_i (M x N, FP64) = A_op(i) (M x K_i) * B_i (K_i x N, FP64) for
// a batch of fields B_i and at most two operators A (M <= 129 rows, K <= 136),
// as three TF32 products A_hi B_hi + A_lo B_hi + A_hi B_lo with FP32
// accumulation in tensor memory (the same 3xTF32 scheme as k_sgemm3): the
// Chebyshev derivative D on the state (y-derivatives), and V^-1 D, V^-1 on the
// nonlinear terms (eigenbasis-in products of FP32-accurate data in the mixed
// form). One persistent CTA of 26 warps per SM, each CTA a contiguous range of
// 32-column tiles (entry-major):
//   * warps 0-16 (converters, warp w = rows 8w..8w+7, lane = column): load the
//     tile's values straight from global memory (coalesced 256-byte rows,
//     rows past K_i and columns past N as zeros) two tiles ahead in registers,
//     with the tile after those brought into L2 by bulk prefetches; split the
//     values into TF32 hi and lo and store them as one 64-row K-major operand
//     (hi rows 0-31, lo rows 32-63) in one of four operand buffers; for
//     M = 129 they also form the FP64 dot products of the operator's last row
//     with their rows;
//   * warp 25 (issuer): issues per K step of 8 two tcgen05.mma.kind::tf32
//     (M = 128) with the operator from tensor memory: A_hi x [B_hi; B_lo]
//     (N = 64: hi*hi into columns 0-31, hi*lo into 32-63) and A_lo x B_hi
//     (N = 32, into columns 0-31), into one of two 64-column accumulator sets;
//   * warps 17-24 (epilogue, two groups of four warps, one per TMEM lane
//     quadrant; group g takes the tiles of accumulator set g): read both
//     accumulators (tcgen05.ld 16x256b), add them in FP32 and store rows
//     < min(M, 128) in FP64 or FP32; row 128 (M = 129) from the converters'
//     dots. They also copy the operator's TF32 parts into tensor memory
//     (tcgen05.st; lane = row, one K element per column): both groups for the
//     first tile, and the group of the first tile of the second operator
//     after the MMAs of the first have completed.
// Every buffer hand-off has its own mbarrier, so no waiter can fall two phases
// behind. Every wait has an iteration limit (a kernel argument); on expiry the
// kernel raises the error flag, every role stops at its next tile, the issuer
// waits (bounded) for its last MMAs, and the CTA frees its TMEM and returns
// (the converters' loads go to registers and the operator copies are
// synchronous: nothing else is in flight into shared or tensor memory).
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
constexpr int kTcConvWarps = kTcKp / 8, kTcEpiWarps = 8;
constexpr int kTcIssuerWarp = kTcConvWarps + kTcEpiWarps;
constexpr int kTcThreads = 32 * (kTcIssuerWarp + 1);  // 832
constexpr int kTcSideDoubles = kTcConvWarps * kTcN;   // partial dots of the last row
constexpr int kTcNB = 4;                               // operand buffers (tiles converted ahead of the MMAs)
// tensor memory: two accumulator sets of (hi*hi + lo*hi, hi*lo) at columns 0
// and 64, the operator's TF32 parts (A from tensor memory, lane = row, one K
// element per column) at 128 and 288 (32-column aligned)
constexpr int kTcTmemCols = 512;
constexpr int kTcAccCols = 2 * kTcN;
constexpr int kTcAHiCol = 2 * kTcAccCols, kTcALoCol = kTcAHiCol + 160;
static_assert(kTcALoCol + kTcKp <= kTcTmemCols, "tensor-memory columns");
constexpr int kTcMaxOps = 2;                          // operators per launch
constexpr int kTcBars = 2 * kTcNB + 2 * 2 + 1;         // full, buffer free; mma done, epilogue done; A ready
constexpr size_t kTcSmem = kTcNB * (size_t)kTcBSize + kTcNB * sizeof(double) * kTcSideDoubles + 8 * kTcBars + 16;

// B[i]: K[i] x N FP64 (row stride ldb), multiplied by operator op[i]; the
// operator parts are packed by tc05_pack_a; xrow: the FP64 row 128 of
// operator 0 when M = 129 (kTcKp values, zero padded), else null
struct Tc05Batch {
  const double* B[kGemmMaxBatch];
  double* C[kGemmMaxBatch];
  int K[kGemmMaxBatch];
  int op[kGemmMaxBatch];
  const float* a_hi[kTcMaxOps];
  const float* a_lo[kTcMaxOps];
  const double* xrow;
  int count;
  int M, N, ldb, ldc;
  int c_f32;     // C holds floats (same element offsets)
  int prefetch;  // every B[i] is 16-byte aligned: rows may be bulk-prefetched into L2
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

// A from tensor memory (lane = row, column = K element), B from shared memory
__device__ __forceinline__ void tc_mma_tf32_ts(uint32_t tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc,
                                               uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc), "r"(0u));
}

// 32 TMEM lanes (the warp's quadrant) x 8 columns: thread = lane, 8 consecutive columns
__device__ __forceinline__ void tc_st32x8(uint32_t taddr, const uint32_t* v) {
  // (no memory clobber: tensor memory only, so global loads may move above it)
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"r"(taddr),
               "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]));
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

// 16 TMEM lanes x 4 repetitions of 256 bits (8 columns): thread (lane % 4,
// lane / 4) receives rows lane / 4 and lane / 4 + 8, columns 8 p + 2 (lane % 4)
// and + 1 of repetition p, in registers 4 p + {0, 1} and 4 p + {2, 3}
__device__ __forceinline__ void tc_ld16x256b_x4(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
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

// *p when c, else 0; volatile, so a prefetch is issued where it stands and is
// waited for only where its value is first used
__device__ __forceinline__ double tc_load_if(const double* p, bool c) {
  double x = 0.0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t@p ld.global.nc.L1::no_allocate.f64 %0, [%1];\n\t}\n"
      : "+d"(x)
      : "l"(p), "r"((int)c));
  return x;
}
#endif

__global__ void __launch_bounds__(kTcThreads, 1) k_tc05_split(const __grid_constant__ Tc05Batch b,
                                                              int* __restrict__ err, int spin) {
#if defined(__CUDA_ARCH__)
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* sB0 = tsm;                                            // kTcNB stacked hi / lo operands
  double* side = reinterpret_cast<double*>(sB0 + kTcNB * kTcBSize);    // kTcNB buffers of partial dots
  uint64_t* bars = reinterpret_cast<uint64_t*>(side + kTcNB * kTcSideDoubles);
  // bars: [0, NB) full (operand + dots of buffer b); [NB, 2NB) buffer b
  // released by the epilogue of its tile (which waited for that tile's MMAs,
  // so the operand has been read too); 2NB + s MMAs of accumulator set s
  // done; 2NB + 2 + s epilogue of set s done; 2NB + 4 A in tensor memory
  constexpr int kFull = 0, kSFree = kTcNB, kMDone = 2 * kTcNB, kEDone = 2 * kTcNB + 2, kAReady = 2 * kTcNB + 4;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + kTcBars);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto bar = [&](int i) { return tc_smem(&bars[i]); };
  if (tid == 0) {
    for (int q = 0; q < kTcNB; ++q) {
      mbar_init(bar(kFull + q), 32 * kTcConvWarps);
      mbar_init(bar(kSFree + q), 32 * kTcEpiWarps / 2);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(bar(kMDone + q), 1);
      mbar_init(bar(kEDone + q), 32 * kTcEpiWarps / 2);
    }
    mbar_init(bar(kAReady), 32 * kTcEpiWarps / 2);
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
  auto fail_now = [&]() {
    *abort_flag = 1;
    atomicOr(err, kErrWaitExpired);
  };
  // entry fields of tile i of this CTA by selects over the parameter arrays
  auto entry_of = [&](int i) { return (t_begin + i) / tiles_n; };
  auto op_of = [&](int e) {
    int op = b.op[0];
#pragma unroll
    for (int q = 1; q < kGemmMaxBatch; ++q)
      if (e == q) op = b.op[q];
    return op;
  };
  auto k_of = [&](int e) {
    int K = b.K[0];
#pragma unroll
    for (int q = 1; q < kGemmMaxBatch; ++q)
      if (e == q) K = b.K[q];
    return K;
  };

  if (warp < kTcConvWarps) {
    // ---------------------------------------------------------------- converters
    const int n = lane, k0 = 8 * warp;
    double xa[8], xb[8];  // two tiles in flight: the loads of tile i + 2 are issued once tile i is stored
    auto fetch = [&](int i, double(&x)[8]) {
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kTcN;
      const double* B = b.B[0];
#pragma unroll
      for (int q = 1; q < kGemmMaxBatch; ++q)
        if (e == q) B = b.B[q];
      const int K = k_of(e);
      const bool cv = n0 + n < b.N;
      const double* src = B + (size_t)k0 * b.ldb + n0 + n;
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = tc_load_if(src + (size_t)j * b.ldb, cv && k0 + j < K);
    };
    // the 8 rows of this warp of tile i into L2 (lane j < 8: row k0 + j, one
    // bulk prefetch of the tile's 256-byte row segment or the part inside N)
    auto prefetch = [&](int i) {
      if (!b.prefetch || lane >= 8) return;
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kTcN;
      const double* B = b.B[0];
#pragma unroll
      for (int q = 1; q < kGemmMaxBatch; ++q)
        if (e == q) B = b.B[q];
      const int K = k_of(e);
      const int cols = b.N - n0 < kTcN ? b.N - n0 : kTcN;  // even: N and n0 are
      if (k0 + lane < K) l2_prefetch(B + (size_t)(k0 + lane) * b.ldb + n0, (unsigned)cols * 8u);
    };
    // tile i from registers x into operand buffer i % NB; then x takes the
    // loads of tile i + 2 (from L2: prefetched a tile earlier)
    auto body = [&](int i, double(&x)[8]) -> bool {
      const int bq = i % kTcNB;
      double dot = 0.0;
      if (b.M > kTcM) {
#pragma unroll
        for (int j = 0; j < 8; ++j) dot = fma(__ldg(b.xrow + k0 + j), x[j], dot);  // xrow is zero padded
      }
      // buffer bq is free once the epilogue of tile i - NB is done with it: it
      // read the dots, after the MMAs that read the operand had completed
      const int ph = ((i / kTcNB) - 1) & 1;
      const bool ok = i < kTcNB || mbar_wait(bar(kSFree + bq), ph, spin);
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        return false;
      }
      unsigned char* sB = sB0 + bq * kTcBSize;
      // one FP64 conversion per value: hi + lo keep 22 of the FP32 value's 24
      // bits, and f - hi is exact in FP32
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float f = (float)x[4 * c + j];
          const float h = tf32_round_dev(f);
          hi[j] = __float_as_uint(h);
          lo[j] = __float_as_uint(tf32_round_dev(f - h));
        }
        *reinterpret_cast<uint4*>(sB + tc05_offset(kTcBRows, n, k0 + 4 * c)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(sB + tc05_offset(kTcBRows, kTcN + n, k0 + 4 * c)) =
            make_uint4(lo[0], lo[1], lo[2], lo[3]);
      }
      side[bq * kTcSideDoubles + warp * kTcN + n] = dot;
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      tc_arrive(bar(kFull + bq));
      if (i + 2 < nt) fetch(i + 2, x);
      if (i + 3 < nt) prefetch(i + 3);
      return true;
    };
    if (nt > 0) fetch(0, xa);
    if (nt > 1) fetch(1, xb);
    if (nt > 2) prefetch(2);
    for (int i = 0; i < nt && !*abort_flag; i += 2) {
      if (!body(i, xa)) break;
      if (i + 1 < nt && !*abort_flag && !body(i + 1, xb)) break;
    }
  } else if (warp < kTcConvWarps + kTcEpiWarps) {
    // ----------------------------------------------------------------- epilogue
    // two groups of 4 warps (one per TMEM lane quadrant, warp % 4), group g
    // taking the tiles i with i % 2 = g (accumulator set g), so each group has
    // two tile periods for its tile. tcgen05.ld 16x256b: thread (t0, t1) =
    // (lane % 4, lane / 4) holds rows t1 and t1 + 8 of a 16-lane half,
    // columns 8p + 2 t0 and + 1 of repetition p, so a quad of threads stores
    // 64 contiguous bytes of a row. The group of the first tile of each
    // operator also copies that operator's TF32 parts into tensor memory.
    const int ew = warp - kTcConvWarps, quad = warp & 3, gq = ew >> 2;
    const int t0 = lane & 3, t1 = lane >> 2;
    const int mt = b.M < kTcM ? b.M : kTcM;
    // columns [c_begin, c_end) (multiples of 8) of both TF32 parts of the
    // operator into this warp's lane quadrant of tensor memory
    auto load_a = [&](int op, int c_begin, int c_end) {
      const int row = 32 * quad + lane;
      const float* hi = (op ? b.a_hi[1] : b.a_hi[0]) + (size_t)row * kTcKp;
      const float* lo = (op ? b.a_lo[1] : b.a_lo[0]) + (size_t)row * kTcKp;
      const uint32_t lanes = (uint32_t)(32 * quad) << 16;
#pragma unroll 3
      for (int c = c_begin; c < c_end; c += 8) {
        uint32_t v[8];
        const float4 h0 = __ldg(reinterpret_cast<const float4*>(hi + c));
        const float4 h1 = __ldg(reinterpret_cast<const float4*>(hi + c + 4));
        v[0] = __float_as_uint(h0.x), v[1] = __float_as_uint(h0.y), v[2] = __float_as_uint(h0.z);
        v[3] = __float_as_uint(h0.w), v[4] = __float_as_uint(h1.x), v[5] = __float_as_uint(h1.y);
        v[6] = __float_as_uint(h1.z), v[7] = __float_as_uint(h1.w);
        tc_st32x8(tmem + lanes + (uint32_t)(kTcAHiCol + c), v);
        const float4 l0 = __ldg(reinterpret_cast<const float4*>(lo + c));
        const float4 l1 = __ldg(reinterpret_cast<const float4*>(lo + c + 4));
        v[0] = __float_as_uint(l0.x), v[1] = __float_as_uint(l0.y), v[2] = __float_as_uint(l0.z);
        v[3] = __float_as_uint(l0.w), v[4] = __float_as_uint(l1.x), v[5] = __float_as_uint(l1.y);
        v[6] = __float_as_uint(l1.z), v[7] = __float_as_uint(l1.w);
        tc_st32x8(tmem + lanes + (uint32_t)(kTcALoCol + c), v);
      }
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
    };
    constexpr int kASplit = 72;  // the two groups' halves of the first load (9 and 8 chunks of 8 columns)
    if (nt > 0) {
      load_a(op_of(entry_of(0)), gq ? kASplit : 0, gq ? kTcKp : kASplit);
      asm volatile("bar.sync 1, %0;\n" ::"n"(32 * kTcEpiWarps) : "memory");  // both halves stored
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      if (gq == 0) tc_arrive(bar(kAReady));
    }
    for (int i = gq; i < nt && !*abort_flag; i += 2) {
      const int e = entry_of(i), op = op_of(e);
      if (i > 0 && op_of(entry_of(i - 1)) != op) {
        // the previous operator is read by every MMA up to tile i - 1
        const bool ok = mbar_wait(bar(kMDone + ((i - 1) & 1)), ((i - 1) >> 1) & 1, spin);
        if (!__all_sync(0xffffffffu, ok)) {
          fail_now();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        load_a(op, 0, kTcKp);
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        tc_arrive(bar(kAReady));
      }
      const int set = i & 1, bq = i % kTcNB;
      bool ok = mbar_wait(bar(kMDone + set), (i >> 1) & 1, spin);
      if (ok && b.M > kTcM) ok = mbar_wait(bar(kFull + bq), (i / kTcNB) & 1, spin);  // the dots
      if (!__all_sync(0xffffffffu, ok)) {  // tcgen05.ld below needs the whole warp
        fail_now();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int n0 = (t_begin + i - e * tiles_n) * kTcN;
      double* C = b.C[0];
#pragma unroll
      for (int q = 1; q < kGemmMaxBatch; ++q)
        if (e == q) C = b.C[q];
#pragma unroll
      for (int hv = 0; hv < 2; ++hv) {
        const uint32_t tbase = tmem + ((uint32_t)(32 * quad + 16 * hv) << 16) + (uint32_t)(set * kTcAccCols);
        uint32_t s0[16], s1[16];
        tc_ld16x256b_x4(tbase, s0);         // hi*hi + lo*hi
        tc_ld16x256b_x4(tbase + kTcN, s1);  // hi*lo
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        const int rowA = 32 * quad + 16 * hv + t1;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          const int col = n0 + 8 * p + 2 * t0;  // even, and N is even: the pair is in range with its first entry
          if (col < b.N) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int row = rowA + 8 * h;
              if (row >= mt) continue;
              // FP32 sum of the two accumulators (the products are FP32-accurate)
              const float x0 = __uint_as_float(s0[4 * p + 2 * h]) + __uint_as_float(s1[4 * p + 2 * h]);
              const float x1 = __uint_as_float(s0[4 * p + 2 * h + 1]) + __uint_as_float(s1[4 * p + 2 * h + 1]);
              if (b.c_f32)
                *reinterpret_cast<float2*>(reinterpret_cast<float*>(C) + (size_t)row * b.ldc + col) =
                    make_float2(x0, x1);
              else
                *reinterpret_cast<double2*>(C + (size_t)row * b.ldc + col) = make_double2((double)x0, (double)x1);
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      if (b.M > kTcM && quad == 0 && n0 + lane < b.N) {
        const double* sd = side + bq * kTcSideDoubles;
        double x = sd[lane];
#pragma unroll
        for (int w = 1; w < kTcConvWarps; ++w) x += sd[w * kTcN + lane];
        C[(size_t)kTcM * b.ldc + n0 + lane] = x;
      }
      tc_arrive(bar(kSFree + bq));
      tc_arrive(bar(kEDone + set));
    }
  } else {
    // ------------------------------------------------------------------- issuer
    if (lane == 0) {
      int issued = 0, a_loads = 0, cur_op = -1;
      constexpr uint32_t lbo_b = kTcBRows * 16;
      const uint64_t db0 = tc05_desc(tc_smem(sB0), lbo_b, 128);
      for (int i = 0; i < nt && !*abort_flag; ++i) {
        const int set = i & 1, bq = i % kTcNB;
        const int e = entry_of(i), op = op_of(e), K = k_of(e);
        if (op != cur_op) {  // the epilogue group of tile i copies the operator into tensor memory
          ++a_loads;
          if (!mbar_wait(bar(kAReady), (a_loads - 1) & 1, spin)) {
            fail_now();
            break;
          }
          cur_op = op;
        }
        if (!mbar_wait(bar(kFull + bq), (i / kTcNB) & 1, spin) ||
            (i >= 2 && !mbar_wait(bar(kEDone + set), ((i - 2) >> 1) & 1, spin))) {
          fail_now();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(set * kTcAccCols);
        // operand buffer bq's descriptor: the start-address field moves by its offset / 16
        const uint64_t db = db0 + (uint64_t)((bq * kTcBSize) >> 4);
        const int ksteps = (K + 7) / 8;  // <= kTcKp / 8
#pragma unroll
        for (int s = 0; s < kTcKp / 8; ++s) {
          if (s >= ksteps) break;
          const uint64_t ob = (2u * s * lbo_b) >> 4;
          tc_mma_tf32_ts(acc, tmem + (uint32_t)(kTcAHiCol + 8 * s), db + ob, tc_idesc_tf32(2 * kTcN),
                         s > 0 ? 1u : 0u);                                                              // hi x [hi; lo]
          tc_mma_tf32_ts(acc, tmem + (uint32_t)(kTcALoCol + 8 * s), db + ob, tc_idesc_tf32(kTcN), 1u);  // lo x hi
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         bar(kMDone + set))
                     : "memory");
        issued = i + 1;
      }
      // no MMA may still run when the CTA frees its tensor memory
      if (issued > 0 && !mbar_wait(bar(kMDone + ((issued - 1) & 1)), ((issued - 1) >> 1) & 1, kDrainPolls))
        fail_now();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)kTcTmemCols));
  }
#endif
}

// Host: rows 0..M-1 of an operator (row-major, ld = ldd) split into TF32 hi /
// lo, 128 rows x kTcKp (rows >= M and K >= k zero), row-major: the layout the
// kernel copies into tensor memory (lane = row).
inline void tc05_pack_a(const double* D, int M, int K, int ldd, float (*tf32)(float), std::vector<float>& hi,
                        std::vector<float>& lo) {
  hi.assign(kTcASize / 4, 0.f);
  lo.assign(kTcASize / 4, 0.f);
  for (int r = 0; r < M && r < kTcM; ++r)
    for (int k = 0; k < K && k < kTcKp; ++k) {
      const double x = D[(size_t)r * ldd + k];
      const float h = tf32((float)x);
      const int off = r * kTcKp + k;
      hi[off] = h;
      lo[off] = tf32((float)(x - (double)h));
    }
}

}  // namespace jsd
