// FP64-accurate products on the int8 tensor cores (Ozaki splitting), for the
// eigenbasis transforms.
//
// C (M x N) = A (M x K) B (K x N), A a constant operator (M, K <= 129), B a
// batch of FP64 fields. Each row i of A and each column j of B is scaled by a
// power of two and cut into 8 signed 7-bit integer slices:
//   a_ik = 2^ea_i sum_p alpha_ikp 2^(-7p),  b_kj = 2^(eb_j + 2) sum_q beta_kjq 2^(-7q),
//   p, q = 1..8. A's digits (packed once on the host) are sign-magnitude,
//   alpha in [-127, 127], of |a| / 2^ea < 1 (56 bits). B's digits (cut on the
//   device every call) are balanced base-128 digits, beta in [-64, 63], of the
//   integer trunc(b 2^(54 - eb)), |.| < 2^54: adding the bias 64 sum_j 128^j
//   makes it a non-negative 56-bit integer whose 7-bit fields minus 64 are the
//   digits, so slicing a value costs one conversion, one 64-bit add and a
//   field extraction per slice (54 bits, against FP64's 53).
// The products alpha_p beta_q are exact int8 tensor-core GEMMs with exact
// int32 accumulation; the pairs with p + q <= 9 (36 products) are kept and
// summed per diagonal d = p + q into 8 int32 accumulators in tensor memory (at
// most 8 pairs x K=128 x 127 x 64 < 2^31), which the epilogue combines in FP64:
//   c_ij = 2^(ea_i - 14) 2^(eb_j + 2) sum_d acc_d 2^(-7 (d - 2)).
// The error bound is of the order of an FP64 GEMM's (the dropped terms and the
// slice remainders are below 2^-56 of |a_i|max |b_j|max per product), so the
// products stay FP64-accurate while the arithmetic runs at int8 tensor rate.
// Tensor rows and K are 128; a 129th row of A (M = 129) or a 129th column
// (K = 129) is applied in FP64 beside the tensor part.
//
// The 8 B slices of a 32-column tile are stacked into one 256-row operand
// (row 32 (q - 1) + column). One MMA per A slice p and K step, with
// N = 32 (9 - p) stacked rows (slices q = 1..9-p) and its accumulator placed
// (p - 1) x 32 TMEM columns on, lands every product (p, q) in the columns of
// diagonal p + q: 32 MMAs of N = 32..256 per tile instead of 36 x 4 narrow
// ones, so the operands are read from shared memory once per wide product.
//
// One persistent CTA of 21 warps per SM, each CTA a contiguous range of
// 32-column tiles:
//   * warps 0-15 (converters, warp w = rows 8w..8w+7, lane = column): load
//     their 8 x 32 block of the tile straight from global memory (a warp reads
//     256 contiguous bytes per row) one tile ahead into registers, exchange
//     the exponents of their partial column maxima through an mbarrier, cut
//     the block into the 8 slices and store them in the canonical K-major
//     core-matrix layout;
//   * warp 16 (issuer): keeps A's 8 slices resident (bulk copy, reloaded when
//     the operator changes), issues the 32 MMAs (kind::i8, M = 128) into one of
//     two accumulator sets of 8 x 32 TMEM columns and commits to an mbarrier;
//   * warps 17-20 (epilogue, TMEM lane quadrant = warp % 4 = row block): per
//     16-column half, read the 8 accumulators (tcgen05.ld, two per wait),
//     combine, scale and add the FP64 extras, write the 32 x 16 block into a
//     128-byte-swizzled shared-memory slot and store it with one TMA store
//     (rows and columns outside C are not written). 21 warps keep at most 6 on
//     a scheduler, which leaves each thread 80 registers.
// A column holding a NaN or an infinity gets a NaN column scale, so the whole
// output column is NaN as in an FP64 product (the slices alone would drop it).
// Every mbarrier wait has an iteration limit (a kernel argument); on expiry
// the kernel raises the error flag, every role stops at its next tile, the
// issuer waits (bounded) for its operand copy and its last MMAs, the epilogue
// warps for their TMA stores, and the CTA frees its TMEM and returns.
#pragma once

#include <cuda.h>  // CUtensorMap (the encoder is reached through the runtime's driver entry point)

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
constexpr int kOzABytes = kOzSlices * kOzASlice;     // 131072
constexpr int kOzBRows = kOzSlices * kOzN;           // stacked B operand rows (256)
constexpr int kOzBBytes = kOzBRows * kOzK;           // 32768
constexpr int kOzTmemCols = 2 * kOzDiags * kOzN;     // 512: two accumulator sets
constexpr int kOzConvWarps = 16, kOzEpiWarps = 4;
constexpr int kOzConvRows = kOzK / kOzConvWarps;  // B rows per converter lane (8)
constexpr int kOzIssuerWarp = kOzConvWarps;
constexpr int kOzThreads = 32 * (kOzConvWarps + 1 + kOzEpiWarps);  // 672
constexpr int kOzOutCols = kOzN / 2;                 // columns per epilogue pass (16 doubles = 128 bytes)
constexpr int kOzOutSlot = 32 * kOzOutCols * 8;      // 4096: one epilogue pass's swizzled output block
// per tile buffer (doubles): column scales, B row 128 (K = 129), row-128 dots (M = 129)
constexpr int kOzSideScale = 0, kOzSideBx = kOzN, kOzSideDot = 2 * kOzN, kOzSideDoubles = 3 * kOzN;
// partial-maximum exponents of a column that is all zero / holds a NaN or an infinity
constexpr int kOzExpZero = -1000, kOzExpBad = 1 << 20;
// shared memory: A slices | B slices | output slots | side data | exchange (exponents, dots) | barriers
constexpr size_t kOzOffB = kOzABytes, kOzOffOut = kOzOffB + kOzBBytes,
                 kOzOffSide = kOzOffOut + 2 * kOzEpiWarps * kOzOutSlot;
constexpr size_t kOzOffPExp = kOzOffSide + 2 * sizeof(double) * kOzSideDoubles;
constexpr size_t kOzOffPDot = kOzOffPExp + 2 * sizeof(int) * kOzConvWarps * kOzN;
constexpr size_t kOzOffBars = kOzOffPDot + 2 * sizeof(double) * kOzConvWarps * kOzN;
constexpr size_t kOzSmem = kOzOffBars + 128 + 1024;  // + alignment of the dynamic shared memory base

// byte offset of element (row r, k) of an R-row int8 operand in the canonical
// K-major layout: core matrix (row group r/8, K chunk k/16) of 8 rows x 16
// bytes at ((k/16) R/8 + r/8) 128; leading byte offset R 16, stride 128
__host__ __device__ __forceinline__ int oz_offset(int R, int r, int k) {
  return ((k >> 4) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 15);
}

// 2^e as a double (|e| well inside the normal range; on the device built from
// the exponent field)
__host__ __device__ __forceinline__ double oz_pow2(int e) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)(e + 1023) << 52);
#else
  return std::ldexp(1.0, e);
#endif
}

// exponent e with |x| < 2^e for every |x| <= m (0 for m = 0), clamped at -900:
// frexp's exponent, on the device read from the exponent field (a subnormal m
// has e <= -1022, so the clamp covers it)
__host__ __device__ __forceinline__ int oz_exponent(double m) {
  if (!(m > 0.0)) return 0;
#if defined(__CUDA_ARCH__)
  const int biased = (int)((unsigned long long)__double_as_longlong(m) >> 52) & 0x7ff;
  const int e = biased == 0 ? -1022 : biased - 1022;
#else
  int e = 0;
  (void)std::frexp(m, &e);
#endif
  return e < -900 ? -900 : e;
}

// Slices of 4 G values already scaled by 2^(56 - e) (|xs| < 2^56), packed
// little-endian: byte j of w[q] (G words) is slice q + 1 of xs[j].
// Sign-magnitude digits (a small value has small digits, so the dropped
// low-order products stay small): the 7-bit fields of trunc(|xs|), negated
// for negative xs. Four elements share a word: their magnitude bytes are
// packed first and the bytes of the negative ones negated together,
// (0x80808080 - W) ^ 0x80808080 being the byte-wise two's complement of bytes
// <= 127 without carries between bytes.
template <int G>
__host__ __device__ __forceinline__ void oz_pack(const double* xs, uint32_t (*w)[G]) {
#pragma unroll
  for (int g = 0; g < G; ++g) {
    unsigned long long a[4];
    uint32_t neg = 0u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double x = xs[4 * g + k];
      a[k] = (unsigned long long)(x < 0.0 ? -x : x);  // truncation toward zero, exact below 2^56
      neg |= (x < 0.0 ? 0xFFu : 0u) << (8 * k);
    }
#pragma unroll
    for (int q = 0; q < kOzSlices; ++q) {
      const int sh = 49 - 7 * q;  // lowest bit of slice q + 1
      uint32_t W = 0u;
#pragma unroll
      for (int k = 0; k < 4; ++k) W |= (uint32_t)((a[k] >> sh) & 127u) << (8 * k);
      const uint32_t nW = (0x80808080u - W) ^ 0x80808080u;
      w[q][g] = W ^ ((W ^ nW) & neg);
    }
  }
}

// 64 sum_{j<8} 128^j: makes trunc(xs) + kOzBias non-negative and below 2^56
// for |xs| < 2^54, with every 7-bit field of the sum equal to its balanced
// digit + 64
constexpr unsigned long long kOzBias = 0x0081020408102040ull;

// Balanced base-128 slices of 4 G integer-valued doubles |xs| < 2^54 (B's
// side), packed little-endian: byte j of w[q] (G words) is digit q + 1 of
// xs[j] (weight 128^(7 - q)) as a signed byte in [-64, 63].
template <int G>
__host__ __device__ __forceinline__ void oz_pack_b(const double* xs, uint32_t (*w)[G], double scale = 1.0) {
#pragma unroll
  for (int g = 0; g < G; ++g) {
    uint32_t lo[4], hi[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const unsigned long long z = (unsigned long long)(long long)(xs[4 * g + k] * scale) + kOzBias;
      lo[k] = (uint32_t)z;
      hi[k] = (uint32_t)(z >> 32);
    }
#pragma unroll
    for (int q = 0; q < kOzSlices; ++q) {
      const int sh = 49 - 7 * q;  // lowest bit of the field of digit q + 1
      uint32_t W = 0u;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        uint32_t f;
        if (sh >= 32)
          f = hi[k] >> (sh - 32);
        else if (sh + 7 <= 32)
          f = lo[k] >> sh;
        else
          f = (lo[k] >> sh) | (hi[k] << (32 - sh));
        W |= (f & 127u) << (8 * k);
      }
      // field f in [0, 127] -> byte f - 64: flip bit 6, and set bit 7 where bit 6 was clear
      w[q][g] = (W ^ 0x40404040u) ^ ((~W & 0x40404040u) << 1);
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

// cmap[i]: 2-D tensor map of entry i's C for TMA stores (inner N doubles,
// outer min(M, 128) rows, row stride ldc), box 16 x 32, 128-byte swizzle
struct OzBatch {
  CUtensorMap cmap[kGemmMaxBatch];
  OzEntry e[kGemmMaxBatch];
  int count;
  int N, ldb, ldc;
  int prefetch;  // every B is 16-byte aligned and ldb even: rows may be bulk-prefetched into L2
};

// one field of entry e by selects (a runtime index into the kernel parameter
// would copy it to local memory; one field is cheaper in registers than the
// whole entry)
#define JSD_OZ_FIELD(name, type)                                   \
  __device__ __forceinline__ type oz_##name(const OzBatch& b, int e) { \
    type r = b.e[0].name;                                          \
    _Pragma("unroll") for (int i = 1; i < kGemmMaxBatch; ++i)      \
      if (e == i) r = b.e[i].name;                                 \
    return r;                                                      \
  }
JSD_OZ_FIELD(B, const double*)
JSD_OZ_FIELD(C, double*)
JSD_OZ_FIELD(a, const int8_t*)
JSD_OZ_FIELD(row_scale, const double*)
JSD_OZ_FIELD(xrow, const double*)
JSD_OZ_FIELD(xcol, const double*)
JSD_OZ_FIELD(M, int)
JSD_OZ_FIELD(K, int)
#undef JSD_OZ_FIELD

#if defined(__CUDA_ARCH__)
// S32 accumulator, signed int8 A and B, both K-major, M = 128, N as given
__host__ __device__ constexpr uint32_t oz_idesc(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kOzM >> 4) << 24);
}

__device__ __forceinline__ void oz_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u));
}

__device__ __forceinline__ void oz_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// *p when c, else 0, as a volatile load: it is issued where it stands (so a
// prefetch does not move up beside the values still being sliced) and is only
// waited for where its value is first used
__device__ __forceinline__ double oz_load_if(const double* p, bool c) {
  double x = 0.0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t@p ld.global.nc.L1::no_allocate.f64 %0, [%1];\n\t}\n"
      : "+d"(x)
      : "l"(p), "r"((int)c));
  return x;
}

// int32 -> double with one FP64 add instead of a conversion: the bit pattern
// 0x43300000:(x ^ 2^31) is the double 2^52 + 2^31 + x (exact below 2^53)
__device__ __forceinline__ double oz_i2d(uint32_t x) {
  return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 4503601774854144.0;
}

#endif

__global__ void __launch_bounds__(kOzThreads, 1) k_oz8_gemm(const __grid_constant__ OzBatch b,
                                                             int* __restrict__ err, int spin) {
#if defined(__CUDA_ARCH__)
  extern __shared__ unsigned char osm_raw[];
  // 1024-byte alignment: the swizzled output slots repeat their pattern every 1024 bytes
  unsigned char* osm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(osm_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = osm;                                        // 8 A slices
  unsigned char* sB = osm + kOzOffB;                              // stacked B slices
  unsigned char* sOut = osm + kOzOffOut;                          // epilogue output slots
  double* side = reinterpret_cast<double*>(osm + kOzOffSide);     // two tile buffers
  int* pexp = reinterpret_cast<int*>(osm + kOzOffPExp);           // [2][16][32] partial-maximum exponents
  double* pdot = reinterpret_cast<double*>(osm + kOzOffPDot);     // [2][16][32] partial row-128 dots
  uint64_t* bars = reinterpret_cast<uint64_t*>(osm + kOzOffBars);
  // bars: 0,1 full (B slices + side data of tile parity); 2,3 mma done;
  // 4,5 epilogue done; 6 A loaded; 7 partial exponents exchanged
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
    mbar_init(bar(7), 32 * kOzConvWarps);
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
    atomicOr(err, kErrWaitExpired);
  };

  if (warp < kOzConvWarps) {
    // ---------------------------------------------------------------- converters
    const int n = lane, k0 = kOzConvRows * warp;
    // tile i = entry e, columns n0..n0+31, walked incrementally (tile t_begin + i);
    // the entry's fields are re-selected only when the entry changes
    int e = t_begin / tiles_n, n0 = (t_begin - e * tiles_n) * kOzN;
    int en = e, n0n = n0;  // the next tile, whose values are prefetched
    int K = oz_K(b, e), M = oz_M(b, e), Kn = K;
    const double* xrow = oz_xrow(b, e);
    const double* Bn = oz_B(b, e);
    // this lane's 8 values (and, for K = 129, row 128) of the tile: loaded one
    // tile ahead, once the previous tile is cut
    double v[kOzConvRows], bx = 0.0;
    auto load_next = [&]() {
      const int kt = Kn < kOzK ? Kn : kOzK;
      const bool cv = n0n + n < b.N;
      const double* src = Bn + (size_t)k0 * b.ldb + n0n + n;
#pragma unroll
      for (int j = 0; j < kOzConvRows; ++j, src += b.ldb) v[j] = oz_load_if(src, cv && k0 + j < kt);
      bx = oz_load_if(Bn + (size_t)kOzK * b.ldb + n0n + n, warp == 0 && cv && Kn > kOzK);
      n0n += kOzN;
      if (n0n >= b.N) {
        n0n = 0;
        ++en;
        if (en < b.count) {
          Kn = oz_K(b, en);
          Bn = oz_B(b, en);
        }
      }
      // the tile after the one just loaded into L2, so that its loads wait
      // for L2 rather than DRAM: lane j < 8 prefetches row k0 + j (warp 0
      // lane 8 row 128), its 256-byte segment or the part inside N
      if (b.prefetch && en < b.count) {
        const int cols = b.N - n0n < kOzN ? b.N - n0n : kOzN;  // even: N and n0n are
        const int row = lane < kOzConvRows ? k0 + lane : (warp == 0 && lane == kOzConvRows ? kOzK : -1);
        if (row >= 0 && row < Kn) l2_prefetch(Bn + (size_t)row * b.ldb + n0n, (unsigned)cols * 8u);
      }
    };
    if (nt > 0) load_next();
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      const int kt = K < kOzK ? K : kOzK;
      double mx = 0.0, dot = 0.0;
      bool bad = false;
#pragma unroll
      for (int j = 0; j < kOzConvRows; ++j) {
        mx = fmax(mx, fabs(v[j]));
        bad |= !isfinite(v[j]);
      }
      if (M > kOzM) {
#pragma unroll
        for (int j = 0; j < kOzConvRows; ++j)
          if (k0 + j < kt) dot = fma(__ldg(xrow + k0 + j), v[j], dot);
      }
      pexp[(buf * kOzConvWarps + warp) * kOzN + n] = bad ? kOzExpBad : (mx > 0.0 ? oz_exponent(mx) : kOzExpZero);
      pdot[(buf * kOzConvWarps + warp) * kOzN + n] = dot;
      tc_arrive(bar(7));
      bool ok = mbar_wait(bar(7), i & 1, spin);
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        break;
      }
      int em = pexp[(buf * kOzConvWarps) * kOzN + n];
#pragma unroll
      for (int w = 1; w < kOzConvWarps; ++w) em = max(em, pexp[(buf * kOzConvWarps + w) * kOzN + n]);
      // warp 0: the row-128 dot of the column (partials summed in warp order),
      // reduced now while few registers are live
      double dsum = 0.0;
      if (warp == 0 && M > kOzM) {
        dsum = pdot[(buf * kOzConvWarps) * kOzN + n];
#pragma unroll
        for (int w = 1; w < kOzConvWarps; ++w) dsum += pdot[(buf * kOzConvWarps + w) * kOzN + n];
      }
      const bool col_bad = em == kOzExpBad;
      const int eb = (em == kOzExpZero || col_bad) ? 0 : em;
      // a NaN / infinity column is sliced as zeros (its NaN scale marks it)
      const double sc = col_bad ? 0.0 : oz_pow2(54 - eb);
      uint32_t wd[kOzSlices][kOzConvRows / 4];
      oz_pack_b<kOzConvRows / 4>(v, wd, sc);
      // the next tile's values are in flight while this one waits for its
      // slice buffer (the loads only land in registers at the next tile's use)
      const double bx_cur = bx;
      if (i + 1 < nt) load_next();
      // the B slices are free once the previous tile's MMAs completed; the
      // side buffer once the epilogue of the tile two back is done (which also
      // frees the accumulator set this tile's MMAs will use)
      ok = (i < 1 || mbar_wait(bar(2 + ((i - 1) & 1)), ((i - 1) >> 1) & 1, spin)) &&
           (i < 2 || mbar_wait(bar(4 + buf), ((i - 2) >> 1) & 1, spin));
      if (!__all_sync(0xffffffffu, ok)) {
        fail_now();
        break;
      }
      static_assert(kOzConvRows == 8, "converter lanes store 8-byte halves of 16-byte core-matrix rows");
#pragma unroll
      for (int q = 0; q < kOzSlices; ++q)
        *reinterpret_cast<uint2*>(sB + oz_offset(kOzBRows, q * kOzN + n, k0)) = make_uint2(wd[q][0], wd[q][1]);
      if (warp == 0) {
        double* sd = side + buf * kOzSideDoubles;
        sd[kOzSideDot + n] = dsum;
        sd[kOzSideScale + n] = col_bad ? __longlong_as_double(0x7ff8000000000000LL) : oz_pow2(eb + 2);
        sd[kOzSideBx + n] = bx_cur;
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      tc_arrive(bar(buf));
      // advance to the next tile
      n0 += kOzN;
      if (n0 >= b.N) {
        n0 = 0;
        ++e;
        if (e < b.count) {
          K = oz_K(b, e);
          M = oz_M(b, e);
          xrow = oz_xrow(b, e);
        }
      }
    }
  } else if (warp == kOzIssuerWarp) {
    // ------------------------------------------------------------------- issuer
    if (lane == 0) {
      const int8_t* cur = nullptr;
      int a_loads = 0, issued = 0;
      for (int i = 0; i < nt && !*abort_flag; ++i) {
        const int buf = i & 1;
        const int t = t_begin + i, e = t / tiles_n;
        const int8_t* a = oz_a(b, e);
        if (a != cur) {
          // the MMAs of the previous tile read the resident slices: let them finish
          if (i > 0 && !mbar_wait(bar(2 + ((i - 1) & 1)), ((i - 1) >> 1) & 1, spin)) {
            fail_now();
            break;
          }
          tc_expect_tx(bar(6), (uint32_t)kOzABytes);
          for (int h = 0; h < 4; ++h)
            tc_bulk_g2s(sA + h * (kOzABytes / 4), a + h * (kOzABytes / 4), (uint32_t)(kOzABytes / 4), bar(6));
          if (!mbar_wait(bar(6), a_loads & 1, spin)) {
            fail_now();
            // the operand copy may still be writing shared memory: let it land
            if (!mbar_wait(bar(6), a_loads & 1, kDrainPolls)) atomicOr(err, kErrWaitExpired);
            break;
          }
          ++a_loads;
          cur = a;
        }
        if (!mbar_wait(bar(buf), (i >> 1) & 1, spin)) {
          fail_now();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        // descriptors at slice 1 / K step 0; the start-address field (bits
        // 0-13, address / 16) of every other operand tile is a constant away
        constexpr uint32_t lbo_a = kOzM * 16, lbo_b = kOzBRows * 16;
        const uint64_t da0 = tc05_desc(tc_smem(sA), lbo_a, 128);
        const uint64_t db0 = tc05_desc(tc_smem(sB), lbo_b, 128);
        const uint32_t acc0 = tmem + (uint32_t)(buf * kOzDiags * kOzN);
#pragma unroll
        for (int ks = 0; ks < kOzK / 32; ++ks)
#pragma unroll
          for (int p = 1; p <= kOzSlices; ++p)
            oz_mma(acc0 + (uint32_t)((p - 1) * kOzN),
                   da0 + (uint64_t)((uint32_t)((p - 1) * kOzASlice + 2 * ks * lbo_a) >> 4),
                   db0 + (uint64_t)((uint32_t)(2 * ks * lbo_b) >> 4), oz_idesc(kOzN * (kOzSlices + 1 - p)),
                   (p == 1 && ks == 0) ? 0u : 1u);
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         bar(2 + buf))
                     : "memory");
        issued = i + 1;
      }
      // no MMA may still run when the CTA frees its tensor memory
      if (issued > 0 && !mbar_wait(bar(2 + ((issued - 1) & 1)), ((issued - 1) >> 1) & 1, kDrainPolls)) fail_now();
    }
  } else {
    // ----------------------------------------------------------------- epilogue
    // warp quad = TMEM lane quadrant = row block; two passes of 16 columns
    const int ew = warp - kOzIssuerWarp - 1, quad = warp & 3;
    const int row = 32 * quad + lane;
    int e = t_begin / tiles_n, n0 = (t_begin - e * tiles_n) * kOzN;
    int M = oz_M(b, e), mt = M < kOzM ? M : kOzM;
    double sa = row < mt ? __ldg(oz_row_scale(b, e) + row) : 0.0;
    double xc = (row < mt && oz_K(b, e) > kOzK) ? __ldg(oz_xcol(b, e) + row) : 0.0;
    for (int i = 0; i < nt && !*abort_flag; ++i) {
      const int buf = i & 1;
      const bool ok = mbar_wait(bar(2 + buf), (i >> 1) & 1, spin) && mbar_wait(bar(buf), (i >> 1) & 1, spin);
      if (!__all_sync(0xffffffffu, ok)) {  // tcgen05.ld below needs the whole warp
        fail_now();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const double* sd = side + buf * kOzSideDoubles;
#pragma unroll 1
      for (int half = 0; half < 2; ++half) {
        const int c0 = kOzOutCols * half;
        unsigned char* slot = sOut + (2 * ew + half) * kOzOutSlot;
        const uint32_t tbase =
            tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(buf * kOzDiags * kOzN) + (uint32_t)c0;
        double r[kOzOutCols];
#pragma unroll
        for (int j = 0; j < kOzOutCols; ++j) r[j] = 0.0;
#pragma unroll
        for (int d = kOzDiags - 1; d >= 1; d -= 2) {  // two loads per wait, highest diagonal first
          uint32_t hi[16], lo[16];
          oz_ld16(tbase + (uint32_t)(d * kOzN), hi);
          oz_ld16(tbase + (uint32_t)((d - 1) * kOzN), lo);
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
          for (int j = 0; j < kOzOutCols; ++j) {
            r[j] = fma(r[j], 0.0078125, oz_i2d(hi[j]));
            r[j] = fma(r[j], 0.0078125, oz_i2d(lo[j]));
          }
        }
        // the slot's previous TMA store must have read it before it is rewritten
        if (lane == 0) tc_bulk_wait_read();
        __syncwarp();
        // 128-byte swizzle: 16-byte chunk j of row `lane` sits at chunk j ^ (lane & 7)
#pragma unroll
        for (int j = 0; j < kOzOutCols; j += 2) {
          const double o0 = fma(xc, sd[kOzSideBx + c0 + j], r[j] * sa * sd[kOzSideScale + c0 + j]);
          const double o1 = fma(xc, sd[kOzSideBx + c0 + j + 1], r[j + 1] * sa * sd[kOzSideScale + c0 + j + 1]);
          *reinterpret_cast<double2*>(slot + lane * 128 + ((((j >> 1) ^ lane) & 7) << 4)) = make_double2(o0, o1);
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        if (lane == 0 && 32 * quad < mt && n0 + c0 < b.N) {
          tc_tma_store_2d(&b.cmap[e], n0 + c0, 32 * quad, slot);
          tc_bulk_commit();
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      if (M > kOzM && ew == 0 && n0 + lane < b.N) oz_C(b, e)[(size_t)kOzM * b.ldc + n0 + lane] = sd[kOzSideDot + lane];
      tc_arrive(bar(4 + buf));
      n0 += kOzN;
      if (n0 >= b.N) {
        n0 = 0;
        ++e;
        if (e < b.count) {
          M = oz_M(b, e);
          mt = M < kOzM ? M : kOzM;
          sa = row < mt ? __ldg(oz_row_scale(b, e) + row) : 0.0;
          xc = (row < mt && oz_K(b, e) > kOzK) ? __ldg(oz_xcol(b, e) + row) : 0.0;
        }
      }
    }
    // this warp's stores read its slots and write C: both done before the CTA ends
    if (lane == 0) tc_bulk_wait_all();
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
      oz_pack<4>(xs, w);
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
