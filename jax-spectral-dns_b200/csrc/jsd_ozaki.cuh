// FP64-accurate products on the int8 tensor cores (Ozaki splitting), for the
// eigenbasis transforms of the mixed-precision form.
//
// C (M x N) = A (M x K) B (K x N), A a constant operator (M, K <= 129), B a
// batch of FP64 fields. Each row i of A and each column j of B is scaled by a
// power of two so that its largest entry is below 1, and the scaled values
// are cut into 8 signed 7-bit integer slices (56 bits):
//   a_ik = 2^ea_i sum_p alpha_ikp 2^(-7p),  b_kj = 2^eb_j sum_q beta_kjq 2^(-7q),
//   alpha, beta in [-127, 127], p, q = 1..8.
// The products alpha_p beta_q are exact int8 tensor-core GEMMs with exact
// int32 accumulation; the pairs with p + q <= 9 (36 GEMMs) are kept and summed
// per diagonal d = p + q into 8 int32 accumulators in tensor memory (at most
// 8 pairs x K=128 x 127^2 < 2^31), which the epilogue combines in FP64:
//   c_ij = 2^(ea_i + eb_j - 14) sum_d acc_d 2^(-7 (d - 2)).
// The error bound is of the order of an FP64 GEMM's (the dropped terms and the
// slice remainders are below 2^-56 of |a_i|max |b_j|max per product), so the
// solves stay FP64-accurate while the arithmetic runs at int8 tensor rate.
// Tensor rows and K are 128; a 129th row of A (M = 129) or a 129th column
// (K = 129) is applied in FP64 beside the tensor part: the converter warps
// form the extra row's dot products from the B values they already hold, and
// the epilogue adds a_i,128 b_128,j.
//
// One persistent CTA of 9 warps per SM, each CTA a contiguous range of
// 32-column tiles:
//   * warps 0-3 (converters): load the 128 x 32 FP64 tile of B (warp w columns
//     8w..8w+7, 4 lanes per column of 32 rows each), find the column scales by
//     shuffles, cut the slices and store them in the canonical K-major
//     core-matrix layout (int8, 16 K per 16-byte row), double-buffered;
//   * warp 8 (issuer): keeps A's 8 slices resident (bulk copy, reloaded when
//     the operator changes), issues 36 x 4 tcgen05.mma.kind::i8 (M = 128,
//     N = 32, K = 32) per tile into one of two accumulator sets of 8 x 32 TMEM
//     columns and commits to an mbarrier;
//   * warps 4-7 (epilogue, TMEM lane quadrant = warp % 4 = row block): read the
//     8 accumulators (tcgen05.ld), combine, scale, add the FP64 extras and
//     store the rows.
// Every mbarrier wait has an iteration limit; on expiry the kernel raises the
// error flag, every role stops at its next tile, the issuer waits (bounded) for
// its last MMAs, and the CTA frees its TMEM and returns.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include "jsd_common.cuh"
#include "jsd_gemm.cuh"
#include "jsd_tc05.cuh"

namespace jsd {

constexpr int kOzSlices = 8;                         // 7-bit slices per operand
constexpr int kOzDiags = kOzSlices;                  // diagonals d = p + q = 2..9
constexpr int kOzM = 128, kOzK = 128, kOzN = 32;     // tensor rows, tensor K, tile columns
constexpr int kOzASlice = kOzM * kOzK;               // bytes per A slice (16384)
constexpr int kOzBSlice = kOzN * kOzK;               // bytes per B slice (4096)
constexpr int kOzABytes = kOzSlices * kOzASlice;     // 131072
constexpr int kOzBBytes = kOzSlices * kOzBSlice;     // 32768 per buffer
constexpr int kOzTmemCols = 2 * kOzDiags * kOzN;     // 512: two accumulator sets
constexpr int kOzConvWarps = 4, kOzEpiWarps = 4;
constexpr int kOzThreads = 32 * (kOzConvWarps + kOzEpiWarps + 1);
// side data per buffer (doubles): column scales, B row 128, extra-row dot products
constexpr int kOzSideScale = 0, kOzSideBx = kOzN, kOzSideDot = 2 * kOzN;
constexpr int kOzSideDoubles = 3 * kOzN;
constexpr size_t kOzSmem = (size_t)kOzABytes + 2 * (size_t)kOzBBytes + 2 * sizeof(double) * kOzSideDoubles + 128;

// byte offset of element (row r, k) of an R-row int8 operand in the canonical
// K-major layout: core matrix (row group r/8, K chunk k/16) of 8 rows x 16
// bytes at ((k/16) R/8 + r/8) 128; leading byte offset R 16, stride 128
__host__ __device__ __forceinline__ int oz_offset(int R, int r, int k) {
  return ((k >> 4) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 15);
}

// 2^e as a double (|e| well inside the normal range)
__host__ __device__ __forceinline__ double oz_pow2(int e) {
#if defined(__CUDA_ARCH__)
  return ldexp(1.0, e);
#else
  return std::ldexp(1.0, e);
#endif
}

// exponent e with |x| < 2^e for every |x| <= m (0 for m = 0)
__host__ __device__ __forceinline__ int oz_exponent(double m) {
  if (!(m > 0.0)) return 0;
  int e = 0;
#if defined(__CUDA_ARCH__)
  (void)frexp(m, &e);
#else
  (void)std::frexp(m, &e);
#endif
  return e < -900 ? -900 : e;
}

// Slices of 16 values already scaled by 2^(56 - e) (|xs| < 2^56), packed
// little-endian: byte j of w[q] (4 words = 16 bytes) is slice q + 1 of xs[j].
__host__ __device__ __forceinline__ void oz_pack16(const double* xs, uint32_t (*w)[4]) {
#pragma unroll
  for (int q = 0; q < kOzSlices; ++q)
#pragma unroll
    for (int t = 0; t < 4; ++t) w[q][t] = 0u;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const long long m = (long long)xs[j];  // truncation toward zero, exact below 2^56
    const unsigned long long a = m < 0 ? (unsigned long long)(-m) : (unsigned long long)m;
    const uint32_t hi = (uint32_t)(a >> 28), lo = (uint32_t)(a & 0xFFFFFFFull);
    const uint32_t neg = m < 0 ? 0xFFu : 0u;
#pragma unroll
    for (int q = 0; q < kOzSlices; ++q) {
      const uint32_t src = q < 4 ? hi : lo;
      const uint32_t v = (src >> (21 - 7 * (q & 3))) & 127u;
      const uint32_t byte = ((v ^ neg) + (neg & 1u)) & 0xFFu;  // two's complement of -v when negative
      w[q][j >> 2] |= byte << (8 * (j & 3));
    }
  }
}

struct OzEntry {
  const int8_t* a;          // 8 slices of the 128 x 128 tensor part, canonical layout
  const double* row_scale;  // 128 entries: 2^(ea_i - 14)
  const double* xrow;       // M = 129: row 128 of A (K values), else null
  const double* xcol;       // K = 129: column 128 of A (128 values), else null
  const double* B;
  double* C;
  int M, K;
};

struct OzBatch {
  OzEntry e[kGemmMaxBatch];
  int count;
  int N, ldb, ldc;
};

// entry e by selects (a runtime index into the kernel parameter would copy the
// parameter array to local memory)
__device__ __forceinline__ OzEntry oz_entry(const OzBatch& b, int e) {
  OzEntry r = b.e[0];
#pragma unroll
  for (int i = 1; i < kGemmMaxBatch; ++i)
    if (e == i) r = b.e[i];
  return r;
}

#if defined(__CUDA_ARCH__)
// S32 accumulator, signed int8 A and B, both K-major, N = 32, M = 128
constexpr uint32_t kOzIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kOzN >> 3) << 17) |
                              ((uint32_t)(kOzM >> 4) << 24);

__device__ __forceinline__ void oz_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kOzIdesc), "r"(acc), "r"(0u));
}

__device__ __forceinline__ void oz_ld32(uint32_t taddr, int* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = (int)r[j];
}

__device__ __forceinline__ void oz_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
#endif

__global__ void __launch_bounds__(kOzThreads, 1) k_oz8_gemm(OzBatch b, int* __restrict__ err) {
#if defined(__CUDA_ARCH__)
  extern __shared__ __align__(1024) unsigned char osm[];
  unsigned char* sA = osm;
  unsigned char* sB = osm + kOzABytes;
  double* side = reinterpret_cast<double*>(osm + kOzABytes + 2 * kOzBBytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(side + 2 * kOzSideDoubles);
  // bars: 0,1 full (B slices ready); 2,3 mma done; 4,5 epilogue done; 6 A loaded
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 8);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto bar = [&](int i) { return tc_smem(&bars[i]); };
  if (tid == 0) {
    mbar_init(bar(0), 32 * kOzConvWarps);
    mbar_init(bar(1), 32 * kOzConvWarps);
    mbar_init(bar(2), 1);
    mbar_init(bar(3), 1);
    mbar_init(bar(4), 32 * kOzEpiWarps);
    mbar_init(bar(5), 32 * kOzEpiWarps);
    mbar_init(bar(6), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc_smem(tslot)),
                 "r"((uint32_t)kOzTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;

  const int tiles_n = (b.N + kOzN - 1) / kOzN;
  const long long total = (long long)tiles_n * b.count;
  const int t_begin = (int)(total * blockIdx.x / gridDim.x);
  const int t_end = (int)(total * (blockIdx.x + 1) / gridDim.x);
  const int nt = t_end - t_begin;
  auto fail_now = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };

  if (warp < kOzConvWarps) {
    // ---------------------------------------------------------------- converters
    // warp w: tile columns 8w..8w+7, lane = (column c = lane % 8, K quarter
    // kq = lane / 8 holding rows 32 kq..32 kq+31); column maxima and the
    // extra row's dot products reduce over the 4 lanes of a column by shuffles
    const int c = lane & 7, kq = lane >> 3, k0 = 32 * kq, n = 8 * warp + c;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      bool ok = i < 2 || mbar_wait(bar(4 + buf), ((i - 2) >> 1) & 1);
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        break;
      }
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kOzN;
      const OzEntry E = oz_entry(b, e);
      const int kt = E.K < kOzK ? E.K : kOzK;
      const int col = n0 + n;
      const bool cv = col < b.N;
      double v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j)
        v[j] = (cv && k0 + j < kt) ? __ldg(E.B + (size_t)(k0 + j) * b.ldb + col) : 0.0;
      double* sd = side + buf * kOzSideDoubles;
      if (kq == 0) sd[kOzSideBx + n] = (E.K > kOzK && cv) ? __ldg(E.B + (size_t)kOzK * b.ldb + col) : 0.0;
      if (E.M > kOzM) {
        double dot = 0.0;
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (k0 + j < kt) dot = fma(__ldg(E.xrow + k0 + j), v[j], dot);
        dot += __shfl_xor_sync(0xffffffffu, dot, 8);
        dot += __shfl_xor_sync(0xffffffffu, dot, 16);
        if (kq == 0) sd[kOzSideDot + n] = dot;
      }
      double mx = 0.0;
#pragma unroll
      for (int j = 0; j < 32; ++j) mx = fmax(mx, fabs(v[j]));
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
      const int eb = oz_exponent(mx);
      if (kq == 0) sd[kOzSideScale + n] = oz_pow2(eb);
      const double sc = oz_pow2(56 - eb);
      unsigned char* dst = sB + buf * kOzBBytes;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        double xs[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) xs[j] = v[16 * h + j] * sc;
        uint32_t w[kOzSlices][4];
        oz_pack16(xs, w);
        const int off = oz_offset(kOzN, n, k0 + 16 * h);
#pragma unroll
        for (int q = 0; q < kOzSlices; ++q)
          *reinterpret_cast<uint4*>(dst + q * kOzBSlice + off) = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      oz_arrive(bar(buf));
    }
  } else if (warp < kOzConvWarps + kOzEpiWarps) {
    // ----------------------------------------------------------------- epilogue
    const int quad = warp & 3, row = 32 * quad + lane;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      // the full wait is already complete (it only orders the converters'
      // side data before the reads below)
      const bool ok = mbar_wait(bar(2 + buf), (i >> 1) & 1) && mbar_wait(bar(buf), (i >> 1) & 1);
      if (!__all_sync(0xffffffffu, ok)) {  // tcgen05.ld below needs the whole warp
        fail_now();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int t = t_begin + i, e = t / tiles_n, n0 = (t - e * tiles_n) * kOzN;
      const OzEntry E = oz_entry(b, e);
      const uint32_t tbase = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(buf * kOzDiags * kOzN);
      double r[32];
      {
        int acc[32];
        oz_ld32(tbase + (uint32_t)((kOzDiags - 1) * kOzN), acc);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int j = 0; j < 32; ++j) r[j] = (double)acc[j];
      }
      for (int d = kOzDiags - 2; d >= 0; --d) {
        int acc[32];
        oz_ld32(tbase + (uint32_t)(d * kOzN), acc);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int j = 0; j < 32; ++j) r[j] = fma(r[j], 0.0078125, (double)acc[j]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      const double* sd = side + buf * kOzSideDoubles;
      const int mt = E.M < kOzM ? E.M : kOzM;
      if (row < mt) {
        const double sa = __ldg(E.row_scale + row);
        const double xc = E.K > kOzK ? __ldg(E.xcol + row) : 0.0;
        double* out = E.C + (size_t)row * b.ldc + n0;
        if (n0 + kOzN <= b.N) {
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const double o0 = fma(xc, sd[kOzSideBx + j], r[j] * sa * sd[kOzSideScale + j]);
            const double o1 = fma(xc, sd[kOzSideBx + j + 1], r[j + 1] * sa * sd[kOzSideScale + j + 1]);
            *reinterpret_cast<double2*>(out + j) = make_double2(o0, o1);
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (n0 + j < b.N) out[j] = fma(xc, sd[kOzSideBx + j], r[j] * sa * sd[kOzSideScale + j]);
        }
      }
      if (E.M > kOzM && quad == 0 && n0 + lane < b.N) {
        E.C[(size_t)kOzM * b.ldc + n0 + lane] = sd[kOzSideDot + lane];
      }
      oz_arrive(bar(4 + buf));
    }
  } else if (lane == 0) {
    // ------------------------------------------------------------------- issuer
    const int8_t* cur = nullptr;
    int a_loads = 0, issued = 0;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      const int t = t_begin + i, e = t / tiles_n;
      const OzEntry E = oz_entry(b, e);
      if (E.a != cur) {
        // the MMAs of the previous tile read the resident slices: let them finish
        if (i > 0 && !mbar_wait(bar(2 + ((i - 1) & 1)), ((i - 1) >> 1) & 1)) {
          fail_now();
          break;
        }
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar(6)),
                     "r"((uint32_t)kOzABytes)
                     : "memory");
        for (int h = 0; h < 4; ++h)
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                  tc_smem(sA + h * (kOzABytes / 4))),
              "l"(E.a + h * (kOzABytes / 4)), "r"((uint32_t)(kOzABytes / 4)), "r"(bar(6))
              : "memory");
        if (!mbar_wait(bar(6), a_loads & 1)) {
          fail_now();
          break;
        }
        ++a_loads;
        cur = E.a;
      }
      if (!mbar_wait(bar(buf), (i >> 1) & 1)) {
        fail_now();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a0 = tc_smem(sA), b0 = tc_smem(sB + buf * kOzBBytes);
      const uint32_t acc0 = tmem + (uint32_t)(buf * kOzDiags * kOzN);
      constexpr uint32_t lbo_a = kOzM * 16, lbo_b = kOzN * 16;
      for (int d = 0; d < kOzDiags; ++d) {  // diagonal p + q = d + 2
        uint32_t accumulate = 0u;
        for (int p = 1; p <= kOzSlices; ++p) {
          const int q = d + 2 - p;
          if (q < 1 || q > kOzSlices) continue;
#pragma unroll
          for (int ks = 0; ks < kOzK / 32; ++ks) {
            const uint64_t da = tc05_desc(a0 + (p - 1) * kOzASlice + 2 * ks * lbo_a, lbo_a, 128);
            const uint64_t db = tc05_desc(b0 + (q - 1) * kOzBSlice + 2 * ks * lbo_b, lbo_b, 128);
            oz_mma(acc0 + (uint32_t)(d * kOzN), da, db, accumulate);
            accumulate = 1u;
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       bar(2 + buf))
                   : "memory");
      issued = i + 1;
    }
    // no MMA may still run when the CTA frees its tensor memory
    if (issued > 0 && !mbar_wait(bar(2 + ((issued - 1) & 1)), ((issued - 1) >> 1) & 1)) fail_now();
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"((uint32_t)kOzTmemCols));
  }
#endif
}

// Host: the tensor part of A (rows < min(M, 128), K < min(K, 128)) as 8 int8
// slices in the canonical layout of a 128 x 128 operand, the row scales
// 2^(ea_i - 14), and the FP64 extras (row 128 when M = 129, column 128 when
// K = 129).
struct OzPackA {
  std::vector<int8_t> slices;
  std::vector<double> row_scale, xrow, xcol;
};

inline void oz_pack_a(const double* A, int M, int K, int lda, OzPackA& out) {
  out.slices.assign(kOzABytes, 0);
  out.row_scale.assign(kOzM, 1.0);
  out.xrow.assign(K > 0 ? K : 1, 0.0);
  out.xcol.assign(kOzM, 0.0);
  const int mt = M < kOzM ? M : kOzM, kt = K < kOzK ? K : kOzK;
  for (int r = 0; r < mt; ++r) {
    double mx = 0.0;
    for (int k = 0; k < kt; ++k) mx = std::fmax(mx, std::fabs(A[(size_t)r * lda + k]));
    const int ea = oz_exponent(mx);
    out.row_scale[r] = oz_pow2(ea - 14);
    const double sc = oz_pow2(56 - ea);
    for (int k0 = 0; k0 < kOzK; k0 += 16) {
      double xs[16];
      for (int j = 0; j < 16; ++j) xs[j] = (k0 + j < kt) ? A[(size_t)r * lda + k0 + j] * sc : 0.0;
      uint32_t w[kOzSlices][4];
      oz_pack16(xs, w);
      for (int q = 0; q < kOzSlices; ++q)
        for (int j = 0; j < 16; ++j)
          out.slices[(size_t)q * kOzASlice + oz_offset(kOzM, r, k0 + j)] =
              (int8_t)(uint8_t)((w[q][j >> 2] >> (8 * (j & 3))) & 0xFFu);
    }
  }
  if (M > kOzM)
    for (int k = 0; k < K; ++k) out.xrow[k] = A[(size_t)kOzM * lda + k];
  if (K > kOzK)
    for (int r = 0; r < mt; ++r) out.xcol[r] = A[(size_t)r * lda + kOzK];
}

}  // namespace jsd
