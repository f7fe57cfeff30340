// Plan management and the C ABI (include/jsd.h) of the velocity-vorticity step.
//
// One RK3/Crank-Nicolson step = 3 stages; each stage launches:
//   1  k_dgemm          D applied to the fields the nonlinear term needs
//   2  k_zinv + k_xmid + k_zfwd   (full / nonlinear equations), or
//      k_linear_terms            (linearised equations)
//   3  k_omega          omega_y of the current state
//   4  k_dgemm          eigenbasis transforms (V^-1 D q, V^-1 [H1, h_g, v, omega])
//   5  k_eigen_update   diagonal solves + influence-matrix correction
//   6  k_mean_flow      (0,0) mean-flow block system
//   7  k_dgemm          back-transform: v, dv/dy, omega_y
//   8  k_reconstruct    u, w from continuity, walls
// and, with constant mass flux, 3 more launches and one copy per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <utility>
#include <string>
#include <vector>

#include "../../include/jsd.h"
#include "jsd_common.cuh"
#include "jsd_fft.cuh"
#include "jsd_gemm.cuh"
#include "jsd_spectral.cuh"
#include "jsd_spectral_sq.cuh"
#include "jsd_tc05.cuh"
#include "jsd_ozaki.cuh"
#include "jsd_adjoint.cuh"

using namespace jsd;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define JSD_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(JSD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

#define JSD_LAUNCHED(name)                                                                  \
  do {                                                                                      \
    cudaError_t e_ = cudaGetLastError();                                                    \
    if (e_ != cudaSuccess)                                                                  \
      return fail(JSD_ERR_CUDA, std::string("launch ") + name + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr double kAlpha[3] = {29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0};
constexpr double kBeta[3] = {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0};
constexpr double kGamma[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
constexpr double kXi[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

constexpr int kXmidZB = 4;

bool smooth_radix(int n) {
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

// sides S of the square FFT lengths S * S with register-resident kernels
constexpr int kSquareSides[] = {3, 4, 5, 7, 10, 14};

int square_side(int n) {
  for (int sd : kSquareSides)
    if (sd * sd == n) return sd;
  return 0;
}

// Call f(std::integral_constant<int, S>) for a supported square side S.
template <typename F>
bool with_square_side(int sd, F&& f) {
  switch (sd) {
    case 3: f(std::integral_constant<int, 3>{}); return true;
    case 4: f(std::integral_constant<int, 4>{}); return true;
    case 5: f(std::integral_constant<int, 5>{}); return true;
    case 7: f(std::integral_constant<int, 7>{}); return true;
    case 10: f(std::integral_constant<int, 10>{}); return true;
    case 14: f(std::integral_constant<int, 14>{}); return true;
    default: return false;
  }
}

// smallest square length with kernels, else the smallest 2,3,5,7-smooth one
int choose_fft_size(int m) {
  const int need = 3 * (m / 2) + 1;
  for (int sd : kSquareSides)
    if (sd * sd >= need) return sd * sd;
  int n = need;
  while (!smooth_radix(n)) ++n;
  return n;
}

// Round an FP32 value to the nearest TF32 value (10 explicit mantissa bits,
// ties away from zero as cvt.rna does).
float tf32_round(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return x;  // inf / nan unchanged
  u = (u + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

// Factor n into supported radices and build the forward twiddle table.
bool build_fft(int n, FftDesc& d, std::vector<double2>& tw) {
  std::vector<int> rs;
  int m = n;
  while (m % 8 == 0) { rs.push_back(8); m /= 8; }
  if (m % 4 == 0) { rs.push_back(4); m /= 4; }
  if (m % 2 == 0) { rs.push_back(2); m /= 2; }
  for (int p : {7, 5, 3})
    while (m % p == 0) { rs.push_back(p); m /= p; }
  if (m != 1 || (int)rs.size() > kMaxFftPasses) return false;
  d.n = n;
  d.passes = (int)rs.size();
  tw.clear();
  int ls = 1;
  for (int p = 0; p < d.passes; ++p) {
    const int r = rs[p];
    d.radix[p] = r;
    d.ls[p] = ls;
    d.twoff[p] = (int)tw.size();
    for (int k = 0; k < ls; ++k)
      for (int t = 1; t < r; ++t) {
        const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)(t * k) /
                                (long double)(ls * r);
        tw.push_back(make_double2((double)cosl(ang), (double)sinl(ang)));
      }
    ls *= r;
  }
  if ((int)tw.size() != n - 1) return false;
  if (tw.empty()) tw.push_back(make_double2(1.0, 0.0));
  return true;
}

}  // namespace

struct jsd_plan {
  jsd_desc desc;
  Geo g;
  FftDesc fx, fz;
  int lda;             // padded leading dimension of the operator matrices
  size_t fdoubles;     // doubles per spectral field (2 ny nk)
  size_t edoubles;     // doubles per eigen-space field (2 (ny-2) nk)
  double dpdx_scale;
  // device operator tables
  double2 *twx = nullptr, *twz = nullptr;
  float2 *twx32 = nullptr, *twz32 = nullptr;
  int nb_max = 1;               // runs the workspace is sized for (g.nb = runs stepped now)
  bool coupling = true;         // false: coupling_term = False terms (perturbation and dual)
  // tcgen05 split-TF32 y-derivatives (mixed form, Ny <= 129): rows computed
  // (min(Ny, 128); for Ny = 129 the y = -1 wall row is left out, which only
  // steady-state stages may do), packed D parts, kernel choice, error flag
  int tc_rows = 0;
  float *tc_ahi = nullptr, *tc_alo = nullptr;
  double* tc_xrow = nullptr;  // Ny = 129: the last row of D (FP64, applied beside the tensor part; zero padded)
  int split_kernel = 0;         // 0: k_sgemm3 (mma.sync), 1: k_tc05_split (tcgen05)
  // split-TF32 eigenbasis-in products of the mixed form's FP32-accurate
  // nonlinear terms: tcgen05 packs (index 0: V^-1 D, 1: V^-1) and row-major
  // TF32 hi / lo parts padded to lda (k_sgemm3); off: FP64-accurate products
  bool split_eig_in = false;
  float *tc_ei_hi[2] = {}, *tc_ei_lo[2] = {};
  float *ei_hi[2] = {}, *ei_lo[2] = {};
  int* errflag = nullptr;       // set by kernels whose bounded waits expired
  int num_sms = 148;
  float split_ms[2] = {};       // autotuner timings of the two split kernels
  // FP64-accurate eigenbasis products on the int8 tensor cores (Ny <= 129;
  // chosen by the mixed form's autotuner, selectable in any plan): slice packs of V^-1 D, V^-1, V and D V (index kOzVinvD ..),
  // the FP64 operator each replaces, and the kernel choice per call site
  int8_t* oz_a[4] = {};
  double *oz_rs[4] = {}, *oz_xr[4] = {}, *oz_xc[4] = {};
  const double* oz_src[4] = {};
  bool oz_ready = false;
  int eig_kernel[3] = {0, 0, 0};  // per GemmSite (eigen sites): 0 DMMA, 1 Ozaki int8
  struct OzMap {
    const double* B = nullptr;
    int N = 0, K = 0, ldb = 0, box_cols = 0, box_rows = 0, swizzle = 0;
    CUtensorMap map;
  };
  static constexpr int kMapCache = 32;
  OzMap oz_maps[kMapCache];  // tensor maps of the operands seen so far (round robin)
  int oz_map_next = 0;
  int wait_limit = kWaitPolls;  // polls before a pipeline wait of the tcgen05 kernels gives up
  float eig_ms[3][2] = {};        // autotuner timings per eigen site: DMMA (best tile), Ozaki
  double* re_run = nullptr;     // Reynolds number per run of a batch (device)
  double* lr_ns = nullptr;      // Linv_ns R_ns per run and stage (row-parallel mean-flow update)
  int gemm_cfg[3] = {2, 2, 2};  // DMMA tile configuration per call site (GemmSite)
  int xmid_variant = 2;         // x-pass kernel (launch_xmid), set at creation, autotuned on request
  float xmid_ms[3] = {};        // autotuner timings of the x-pass variants (0: not timed)
  float tune_ms[3][kDgemmConfigs] = {};  // autotuner timings per site and configuration (0: not timed)
  int sqx = 0, sqz = 0;  // square sides of the FFT lengths (0: shared-memory kernels)
  double2 *tsqx = nullptr, *tsqz = nullptr;  // w_N^e, e = 0..N-1, for the square kernels
  float2 *tsqx32 = nullptr, *tsqz32 = nullptr;
  float *Dhi = nullptr, *Dlo = nullptr;  // TF32 split of D (mixed precision)
  bool mixed = false;
  double *Dm = nullptr, *VinvD = nullptr, *Vinv = nullptr, *Vfull = nullptr, *DVfull = nullptr;
  double *lam = nullptr, *sgn = nullptr, *c0 = nullptr, *cN = nullptr, *w0 = nullptr, *wN = nullptr;
  double *yw = nullptr, *rhs_ns = nullptr, *lhs_inv_ns = nullptr, *ub = nullptr, *dub = nullptr;
  // workspace
  double2 *Dfld = nullptr;     // 3 fields: D u, D v, D w
  void *inter = nullptr;       // 9 (18 for the dual) z-transformed lines per (y, kx >= 0)
  void *out3 = nullptr;        // 3 x-transformed products per (y, kx >= 0)
  double2 *q = nullptr, *H1 = nullptr, *hg = nullptr, *om = nullptr, *dvn = nullptr, *tmp = nullptr;
  double2 *conv = nullptr;     // 3 stages x 2 ny
  double2 *uw00 = nullptr;     // 2 ny
  double *X1 = nullptr, *T = nullptr, *hv_old = nullptr, *hg_old = nullptr, *vnt = nullptr, *omnt = nullptr;
  double *vnt_alt = nullptr, *omnt_alt = nullptr;  // ping-pong partners of vnt / omnt
  double *partial = nullptr, *scal = nullptr;
  size_t ws_bytes = 0;
  std::vector<void*> allocs;
  const double2* history = nullptr;
  int n_history = 0;
  // source terms added in every stage (jsd_set_source; caller-owned, device)
  const double2 *src_hv = nullptr, *src_hg = nullptr, *src_00 = nullptr;
  // Discrete adjoint of the linearised perturbation step (jsd_step_adjoint):
  // transposed operators (padded to lda), transposed mean-flow matrices per
  // stage, and small cotangent buffers of the (0,0) system
  double *VinvD_T = nullptr, *Vinv_T = nullptr, *Vfull_T = nullptr, *DVfull_T = nullptr, *D_T = nullptr;
  double *lr_T = nullptr, *li_T = nullptr;
  double2 *adj_conv = nullptr, *adj_x00 = nullptr, *adj_ub = nullptr;
  // Carried between stages of one jsd_step call: vnt / omnt hold V^-1 v and
  // V^-1 omega_y of the current state, dvn holds dv/dy of the current state.
  bool ev_valid = false, om_valid = false, dv_valid = false;
  // optional per-kernel-class timing with CUDA events (jsd_profile_*)
  bool profiling = false;
  std::vector<cudaEvent_t> ev_free;
  struct Rec { int cls; cudaEvent_t a, b; double work; };
  std::vector<Rec> recs;
};

namespace {

int dev_alloc(jsd_plan* p, void** ptr, size_t bytes) {
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) return fail(JSD_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  p->allocs.push_back(*ptr);
  p->ws_bytes += bytes;
  return 0;
}

template <typename T>
int upload(jsd_plan* p, T** dst, const T* src, size_t count) {
  int rc = dev_alloc(p, (void**)dst, count * sizeof(T));
  if (rc) return rc;
  JSD_CUDA(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// rows x cols host matrix (row-major) -> device with leading dimension lda, zero padded
int upload_padded(jsd_plan* p, double** dst, const double* src, int rows, int cols, int lda) {
  std::vector<double> buf((size_t)rows * lda, 0.0);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) buf[(size_t)r * lda + c] = src[(size_t)r * cols + c];
  return upload(p, dst, buf.data(), buf.size());
}

cudaEvent_t take_event(jsd_plan* p) {
  if (!p->ev_free.empty()) {
    cudaEvent_t e = p->ev_free.back();
    p->ev_free.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Brackets one launch of kernel class `cls` with events when profiling.
struct ProfScope {
  jsd_plan* p;
  int cls;
  double work;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  ProfScope(jsd_plan* p_, int cls_, double work_, cudaStream_t s_) : p(p_), cls(cls_), work(work_), s(s_) {
    if (p->profiling) {
      a = take_event(p);
      cudaEventRecord(a, s);
    }
  }
  ~ProfScope() {
    if (p->profiling) {
      cudaEvent_t b = take_event(p);
      cudaEventRecord(b, s);
      p->recs.push_back({cls, a, b, work});
    }
  }
};

double gemm_flops(const GemmBatch& b) {
  double f = 0;
  for (int i = 0; i < b.count; ++i) f += 2.0 * b.e[i].M * (double)b.e[i].K * b.N;
  return f;
}

// GEMM call sites with their own tile configuration
enum GemmSite { kSiteDfield = 0, kSiteEigIn = 1, kSiteEigOut = 2, kGemmSites = 3 };

int launch_gemm_cfg(const jsd_plan* p, const GemmBatch& b, int max_m, int cfg, cudaStream_t s) {
  with_dgemm_cfg(cfg, [&](auto c) {
    using Cfg = decltype(c);
    const dim3 grid((b.N + Cfg::BN - 1) / Cfg::BN, (max_m + Cfg::BM - 1) / Cfg::BM, b.count);
    k_dgemm_t<Cfg><<<grid, Cfg::THREADS, Cfg::BYTES, s>>>(b);
  });
  JSD_LAUNCHED("k_dgemm");
  return 0;
}

int launch_gemm(const jsd_plan* p, const GemmBatch& b, int max_m, GemmSite site, cudaStream_t s);

GemmBatch gemm_batch(const jsd_plan* p);
void add_entry(GemmBatch& b, const double* A, const double* B, double* C, int M, int K, double alpha = 1.0);

// 2-D tensor map of a row-major FP64 matrix (defined below)
int oz_tensor_map(jsd_plan* p, const double* B, int N, int rows, int ldb, int box_cols, int box_rows, bool swizzle128,
                  CUtensorMap* out);

// Split-TF32 products on tcgen05: dst[i] = A_op[i] src[i] (K[i] rows of
// src, M <= 129 rows of the operators; row 128 of operator 0 in FP64 from
// xrow), operators given as tc05_pack_a parts; c_f32: dst holds floats.
int launch_tc05(jsd_plan* p, const float* const* a_hi, const float* const* a_lo, const int* op,
                const double* const* src, const int* K, double* const* dst, int count, int M, const double* xrow,
                cudaStream_t s, bool c_f32 = false) {
  if (count < 1 || count > kGemmMaxBatch || M < 1 || M > kTcM + 1 || (M > kTcM && !xrow))
    return fail(JSD_ERR_ARG, "tcgen05 split product: bad batch");
  Tc05Batch b;
  memset(&b, 0, sizeof(b));
  b.N = 2 * p->g.nk * p->g.nb;
  b.M = M;
  b.ldb = b.ldc = b.N;
  b.xrow = xrow;
  b.c_f32 = c_f32 ? 1 : 0;
  b.prefetch = (b.ldb % 2) == 0 ? 1 : 0;
  double flops = 0.0;
  for (int i = 0; i < count; ++i) {
    if (op[i] < 0 || op[i] >= kTcMaxOps || K[i] < 1 || K[i] > kTcKp || !a_hi[op[i]] || !a_lo[op[i]])
      return fail(JSD_ERR_ARG, "tcgen05 split product: bad entry");
    b.B[i] = src[i];
    b.C[i] = dst[i];
    b.K[i] = K[i];
    b.op[i] = op[i];
    if (reinterpret_cast<uintptr_t>(src[i]) % 16) b.prefetch = 0;
    flops += 2.0 * M * (double)K[i] * b.N;
  }
  for (int o = 0; o < kTcMaxOps; ++o) {
    b.a_hi[o] = a_hi[o];
    b.a_lo[o] = a_lo[o];
  }
  b.count = count;
  const int tiles = (b.N + kTcN - 1) / kTcN * b.count;
  ProfScope ps(p, JSD_PROF_SGEMM, flops, s);
  k_tc05_split<<<tiles < p->num_sms ? tiles : p->num_sms, kTcThreads, kTcSmem, s>>>(b, p->errflag, p->wait_limit);
  JSD_LAUNCHED("k_tc05_split");
  return 0;
}

// D * f on tcgen05 (all Ny <= 129 rows of D; row 128 in FP64)
int launch_tc05_dfield(jsd_plan* p, const double* const* src, double* const* dst, int count, cudaStream_t s) {
  const float* hi[kTcMaxOps] = {p->tc_ahi, p->tc_ahi};
  const float* lo[kTcMaxOps] = {p->tc_alo, p->tc_alo};
  int op[kGemmMaxBatch] = {}, K[kGemmMaxBatch] = {};
  for (int i = 0; i < count && i < kGemmMaxBatch; ++i) K[i] = p->g.ny;
  return launch_tc05(p, hi, lo, op, src, K, dst, count, p->tc_rows, p->tc_xrow, s);
}

// Split-TF32 eigenbasis-in products of the nonlinear terms (mixed form):
// X1 = V^-1 D q, T_0 = V^-1 H1, T_1 = V^-1 h_g (interior rows, stored in
// FP32), on tcgen05 or k_sgemm3 as the plan's split-kernel choice says.
int launch_split_eig_in(jsd_plan* p, cudaStream_t s) {
  const int ny = p->g.ny, ni = ny - 2;
  const size_t E = p->edoubles, rowd = 2 * (size_t)p->g.nk * p->g.nb;
  const double* src[3] = {(const double*)p->q, (const double*)p->H1 + rowd, (const double*)p->hg + rowd};
  double* dst[3] = {p->X1, p->T, p->T + E};
  const int K[3] = {ny, ni, ni};
  const int op[3] = {0, 1, 1};
  if (p->split_kernel == 1 && p->tc_rows)
    return launch_tc05(p, p->tc_ei_hi, p->tc_ei_lo, op, src, K, dst, 3, ni, nullptr, s, true);
  SplitGemmBatch b;
  memset(&b, 0, sizeof(b));
  b.c_f32 = 1;
  b.N = 2 * p->g.nk * p->g.nb;
  b.lda = p->lda;
  b.ldb = b.N;
  b.ldc = b.N;
  double flops = 0.0;
  for (int i = 0; i < 3; ++i) {
    SplitGemmEntry& e = b.e[b.count++];
    e.Ahi = p->ei_hi[op[i]];
    e.Alo = p->ei_lo[op[i]];
    e.B = src[i];
    e.C = dst[i];
    e.M = ni;
    e.K = K[i];
    flops += 2.0 * ni * (double)K[i] * b.N;
  }
  ProfScope ps(p, JSD_PROF_SGEMM, flops, s);
  const dim3 grid((b.N + Sgemm3Smem::BN - 1) / Sgemm3Smem::BN, 1, b.count);
  k_sgemm3<<<grid, Sgemm3Smem::THREADS, Sgemm3Smem::BYTES, s>>>(b);
  JSD_LAUNCHED("k_sgemm3");
  return 0;
}

// y-derivatives D * f of up to kGemmMaxBatch fields: FP64 DMMA, or 3xTF32 in
// the mixed-precision mode (mma.sync, or tcgen05 when the plan chose it and
// the call allows its rows: all rows for Ny <= 128; for Ny = 129 only calls
// whose wall-row derivatives are never used, `walls_free`)
int launch_dfield(jsd_plan* p, const double* const* src, double* const* dst, int count, cudaStream_t s,
                  bool walls_free = false, int force_split = -1) {
  const int ny = p->g.ny;
  if (!p->mixed) {
    GemmBatch b = gemm_batch(p);
    for (int i = 0; i < count; ++i) add_entry(b, p->Dm, src[i], dst[i], ny, ny, 1.0);
    return launch_gemm(p, b, ny, kSiteDfield, s);
  }
  const int kernel = force_split >= 0 ? force_split : p->split_kernel;
  (void)walls_free;  // the tcgen05 kernel computes every row, the y = -1 wall row in FP64
  if (kernel == 1 && p->tc_rows) return launch_tc05_dfield(p, src, dst, count, s);
  SplitGemmBatch b;
  memset(&b, 0, sizeof(b));
  b.N = 2 * p->g.nk * p->g.nb;
  b.lda = p->lda;
  b.ldb = b.N;
  b.ldc = b.N;
  for (int i = 0; i < count; ++i) {
    SplitGemmEntry& e = b.e[b.count++];
    e.Ahi = p->Dhi;
    e.Alo = p->Dlo;
    e.B = src[i];
    e.C = dst[i];
    e.M = ny;
    e.K = ny;
  }
  ProfScope ps(p, JSD_PROF_SGEMM, 2.0 * ny * (double)ny * b.N * count, s);
  const dim3 grid((b.N + Sgemm3Smem::BN - 1) / Sgemm3Smem::BN, 1, b.count);
  k_sgemm3<<<grid, Sgemm3Smem::THREADS, Sgemm3Smem::BYTES, s>>>(b);
  JSD_LAUNCHED("k_sgemm3");
  return 0;
}

GemmBatch gemm_batch(const jsd_plan* p) {
  GemmBatch b;
  memset(&b, 0, sizeof(b));
  b.N = 2 * p->g.nk * p->g.nb;
  b.lda = p->lda;
  b.ldb = b.N;
  b.ldc = b.N;
  return b;
}

void add_entry(GemmBatch& b, const double* A, const double* B, double* C, int M, int K, double alpha) {
  GemmEntry& e = b.e[b.count++];
  e.A = A;
  e.B = B;
  e.C = C;
  e.M = M;
  e.K = K;
  e.alpha = alpha;
}

int launch_gemm(const jsd_plan* p, const GemmBatch& b, int max_m, GemmSite site, cudaStream_t s) {
  ProfScope ps(const_cast<jsd_plan*>(p), JSD_PROF_GEMM, gemm_flops(b), s);
  return launch_gemm_cfg(p, b, max_m, p->gemm_cfg[site], s);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (null when
// the driver does not provide it)
using EncodeTiledFn = decltype(&cuTensorMapEncodeTiled);
EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  });
  return fn;
}

// 2-D tensor map of a row-major FP64 matrix (N doubles per row, `rows` rows,
// row stride ldb), box box_cols x box_rows, zero fill outside on loads and no
// writes outside on stores, optionally with the 128-byte swizzle; cached per plan
int oz_tensor_map(jsd_plan* p, const double* B, int N, int rows, int ldb, int box_cols, int box_rows, bool swizzle128,
                  CUtensorMap* out) {
  for (const auto& m : p->oz_maps)
    if (m.B == B && m.N == N && m.K == rows && m.ldb == ldb && m.box_cols == box_cols && m.box_rows == box_rows &&
        m.swizzle == (int)swizzle128) {
      *out = m.map;
      return 0;
    }
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc) return fail(JSD_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  auto& slot = p->oz_maps[p->oz_map_next];
  p->oz_map_next = (p->oz_map_next + 1) % jsd_plan::kMapCache;
  const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ldb * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(&slot.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(B), dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    slot.B = nullptr;
    return fail(JSD_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  }
  slot.B = B;
  slot.N = N;
  slot.K = rows;
  slot.ldb = ldb;
  slot.box_cols = box_cols;
  slot.box_rows = box_rows;
  slot.swizzle = (int)swizzle128;
  *out = slot.map;
  return 0;
}

// The eigenbasis products of a batch on the int8 tensor cores (k_oz8_gemm);
// every entry's operator must be one of the packed ones.
int launch_ozaki(const jsd_plan* pc, const GemmBatch& b, cudaStream_t s) {
  jsd_plan* p = const_cast<jsd_plan*>(pc);  // the tensor-map cache
  OzBatch o;
  memset(&o, 0, sizeof(o));
  o.N = b.N;
  o.ldb = b.ldb;
  o.ldc = b.ldc;
  o.prefetch = (b.ldb % 2) == 0 ? 1 : 0;
  for (int i = 0; i < b.count; ++i) {
    const GemmEntry& g = b.e[i];
    int k = 0;
    while (k < 4 && p->oz_src[k] != g.A) ++k;
    if (k == 4 || g.alpha != 1.0) return fail(JSD_ERR_STATE, "operator has no int8 slice pack");
    if (reinterpret_cast<uintptr_t>(g.C) % 16 || b.ldc % 2 || b.N % 2)
      return fail(JSD_ERR_STATE, "int8 eigenbasis product needs 16-byte aligned output rows");
    // TMA stores of 16 x 32 output blocks into the tensor part's rows (< 128)
    int rc = oz_tensor_map(p, g.C, b.N, g.M < kOzM ? g.M : kOzM, b.ldc, kOzOutCols, 32, true, &o.cmap[o.count]);
    if (rc) return rc;
    OzEntry& e = o.e[o.count++];
    e.a = p->oz_a[k];
    e.row_scale = p->oz_rs[k];
    e.xrow = p->oz_xr[k];
    e.xcol = p->oz_xc[k];
    e.B = g.B;
    e.C = g.C;
    e.M = g.M;
    e.K = g.K;
    if (reinterpret_cast<uintptr_t>(g.B) % 16) o.prefetch = 0;
  }
  const long long tiles = (long long)((o.N + kOzN - 1) / kOzN) * o.count;
  ProfScope ps(const_cast<jsd_plan*>(p), JSD_PROF_GEMM, gemm_flops(b), s);
  k_oz8_gemm<<<(int)std::min<long long>(tiles, p->num_sms), kOzThreads, kOzSmem, s>>>(o, p->errflag,
                                                                                       p->wait_limit);
  JSD_LAUNCHED("k_oz8_gemm");
  return 0;
}

// eigenbasis in / out products: DMMA, or the Ozaki int8 kernel where the plan
// chose it for the site (force: -1 the plan's choice, 0 DMMA, 1 Ozaki)
int launch_eig(const jsd_plan* p, const GemmBatch& b, int max_m, GemmSite site, cudaStream_t s, int force = -1) {
  const int k = force >= 0 ? force : p->eig_kernel[site];
  if (k == 1 && p->oz_ready) return launch_ozaki(p, b, s);
  return launch_gemm(p, b, max_m, site, s);
}

int grid_for(size_t total, int block) {
  size_t g = (total + block - 1) / block;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g < 1 ? 1 : g);
}

// Geometry seen by kernels that work plane by plane: one plane per (y, run).
Geo planes_of(const Geo& g) {
  Geo gp = g;
  gp.ny = g.ny * g.nb;
  return gp;
}

// h_v = -D q - k^2 H1 (only for the nonlinear-term hook)
__global__ void k_assemble_hv(Geo g, const double2* __restrict__ dq, const double2* __restrict__ h1,
                              double2* __restrict__ hv) {
  const size_t total = (size_t)g.ny * g.nk;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(t % g.nk);
    const int ix = r / g.mz, iz = r - (r / g.mz) * g.mz;
    const double kx = kx_of(g, ix), kz = kz_of(g, iz);
    const double k2 = kx * kx + kz * kz;
    hv[t] = make_double2(-dq[t].x - k2 * h1[t].x, -dq[t].y - k2 * h1[t].y);
  }
}

template <typename C>
int transforms(jsd_plan* p, const double2* state, const double2* uhist, double2* conv, cudaStream_t s);

// nonlinear terms of `state` into p->q, p->H1, p->hg and conv00 slot `stage`
int nonlinear(jsd_plan* p, const double2* state, const double2* uhist, int stage, cudaStream_t s) {
  const Geo& g = p->g;
  const Geo gp = planes_of(g);
  const size_t fs = (size_t)gp.ny * g.nk;
  const double2* u = state;
  const double2* v = state + fs;
  const double2* w = state + 2 * fs;
  double2* conv = p->conv + (size_t)stage * 2 * gp.ny;
  const bool linear = p->desc.linearise && p->desc.kind != JSD_KIND_NS;
  if (p->desc.kind == JSD_KIND_DUAL && !linear && !uhist)
    return fail(JSD_ERR_STATE, "dual step needs the forward state (jsd_set_history)");
  const double2* dv_in = p->dv_valid ? p->dvn : p->Dfld + fs;
  if (linear) {
    if (!p->dv_valid) {
      const double* src[1] = {(const double*)v};
      double* dst[1] = {(double*)(p->Dfld + fs)};
      int rc = launch_dfield(p, src, dst, 1, s);
      if (rc) return rc;
    }
    const int blk = 256;
    ProfScope ps(p, JSD_PROF_LINEAR, sizeof(double2) * 7.0 * fs, s);
    if (p->desc.kind == JSD_KIND_PERTURBATION)
      k_linear_terms<kPerturbation><<<grid_for(fs, blk), blk, 0, s>>>(gp, u, v, w, dv_in, p->ub, p->dub,
                                                                      p->q, p->H1, p->hg, conv);
    else
      k_linear_terms<kDual><<<grid_for(fs, blk), blk, 0, s>>>(gp, u, v, w, dv_in, p->ub, p->dub, p->q,
                                                              p->H1, p->hg, conv);
    JSD_LAUNCHED("k_linear_terms");
    return 0;
  }
  const bool dual = p->desc.kind == JSD_KIND_DUAL;
  {
    const double* src[6];
    double* dst[6];
    int cnt = 0;
    for (int c = 0; c < 3; ++c) {
      if (c == 1 && p->dv_valid) continue;  // dv/dy of the state is already in dvn
      src[cnt] = (const double*)(state + c * fs);
      dst[cnt++] = (double*)(p->Dfld + c * fs);
    }
    if (dual)
      for (int c = 0; c < 3; ++c) {
        src[cnt] = (const double*)(uhist + c * fs);
        dst[cnt++] = (double*)(p->Dfld + (3 + c) * fs);
      }
    // after the first stage of a call the state comes out of k_reconstruct,
    // which zeroes u, v, w on the wall rows: every product that multiplies a
    // wall-row derivative of u or w then vanishes (dv/dy is carried in dvn)
    int rc = launch_dfield(p, src, dst, cnt, s, p->dv_valid && !dual);
    if (rc) return rc;
  }
  return p->mixed ? transforms<float2>(p, state, uhist, conv, s) : transforms<double2>(p, state, uhist, conv, s);
}

// x-pass variants: 0 register square FFT (S lanes per line), 1 half-split
// register FFT (2 S lanes per line, even S, not the dual), 2 shared-memory FFT.
// The S-lane form holds S points x 7 (11 for the dual) products per lane, more
// than the register file in FP64 beyond S = 7.
bool xmid_available(const jsd_plan* p, int v) {
  const bool dual = p->desc.kind == JSD_KIND_DUAL;
  const int S = p->sqx;
  if (v == 0) return S && (p->mixed || S <= 7);
  if (v == 1) return S && S % 2 == 0 && !dual;
  if (v == 2) return smooth_radix(p->g.px) && (size_t)kXmidZB * p->g.px <= (size_t)kXmidEPT * kXmidThreads;
  return false;
}

int default_xmid_variant(const jsd_plan* p) {
  if (p->mixed && xmid_available(p, 0)) return 0;
  if (xmid_available(p, 1)) return 1;
  if (xmid_available(p, 0)) return 0;
  return 2;
}

template <typename C>
int launch_xmid(jsd_plan* p, int variant, C* inter, C* out3, cudaStream_t s) {
  const Geo g = planes_of(p->g);
  const int ny = g.ny;
  const bool dual = p->desc.kind == JSD_KIND_DUAL;
  const double lam = (p->desc.kind == JSD_KIND_NS || !p->desc.linearise) ? 1.0 : 0.0;
  const bool pert = p->desc.kind == JSD_KIND_PERTURBATION;
  const double* ub = pert ? p->ub : nullptr;
  const double* dub = pert ? p->dub : nullptr;
  if (!xmid_available(p, variant)) return fail(JSD_ERR_ARG, "x-pass variant not available for this plan");
  if (variant == 2) {
    const C* twx = p->mixed ? (const C*)p->twx32 : (const C*)p->twx;
    const size_t sm = XmidSmem<C, kXmidZB>::bytes(g);
    const dim3 grid((g.pz + kXmidZB - 1) / kXmidZB, ny);
    if (dual)
      k_xmid_dual<C, kXmidZB><<<grid, kXmidThreads, sm, s>>>(g, p->fx, twx, inter, out3, p->ub, p->dub);
    else
      k_xmid<C, kXmidZB><<<grid, kXmidThreads, sm, s>>>(g, p->fx, twx, inter, out3, ub, dub, lam);
    JSD_LAUNCHED("k_xmid");
    return 0;
  }
  const C* tab = p->mixed ? (const C*)p->tsqx32 : (const C*)p->tsqx;
  with_square_side(p->sqx, [&](auto side) {
    constexpr int S = decltype(side)::value;
    if (variant == 0) {
      constexpr int ZC = XmidSq<C, S>::ZC;
      const dim3 grid((g.pz + ZC - 1) / ZC, ny);
      if (dual)
        k_xmid_dual_sq<C, S><<<grid, kSqWarps * 32, XmidSq<C, S>::smem(g, 2 * kZinvLines), s>>>(
            g, tab, inter, out3, p->ub, p->dub);
      else
        k_xmid_sq<C, S><<<grid, kSqWarps * 32, XmidSq<C, S>::smem(g, kZinvLines), s>>>(g, tab, inter, out3, ub,
                                                                                      dub, lam);
    } else if constexpr (S % 2 == 0) {
      constexpr int ZC = XmidH2<C, S>::ZC;
      const dim3 grid((g.pz + ZC - 1) / ZC, ny);
      k_xmid_h2<C, S><<<grid, kSqWarps * 32, XmidH2<C, S>::smem(g, kZinvLines), s>>>(g, tab, inter, out3, ub, dub,
                                                                                    lam);
    }
  });
  JSD_LAUNCHED("k_xmid_sq");
  return 0;
}

template <typename C>
int transforms(jsd_plan* p, const double2* state, const double2* uhist, double2* conv, cudaStream_t s) {
  const Geo g = planes_of(p->g);
  const size_t fs = (size_t)g.ny * g.nk;
  const int ny = g.ny;
  const bool dual = p->desc.kind == JSD_KIND_DUAL;
  const int nsets = dual ? 2 : 1;
  const int K1 = g.kx_max + 1;
  const C* twx = p->mixed ? (const C*)p->twx32 : (const C*)p->twx;
  const C* twz = p->mixed ? (const C*)p->twz32 : (const C*)p->twz;
  C* inter = static_cast<C*>(p->inter);
  C* out3 = static_cast<C*>(p->out3);
  {
    ZinvSrc src;
    src.nsets = nsets;
    for (int c = 0; c < 3; ++c) {
      src.f[c] = state + c * fs;
      src.f[3 + c] = (c == 1 && p->dv_valid) ? p->dvn : p->Dfld + c * fs;
      if (dual) {
        src.f[6 + c] = uhist + c * fs;
        src.f[9 + c] = p->Dfld + (3 + c) * fs;
      }
    }
    const int nl = kZinvLines * nsets;
    const size_t sm = sizeof(C) * ((size_t)g.pz + 2 * (size_t)nl * fline(g.pz));
    const double bytes = sizeof(double2) * 6.0 * nsets * fs + sizeof(C) * (double)nl * ny * K1 * g.pz;
    ProfScope ps(p, JSD_PROF_ZINV, bytes, s);
    if (p->sqz) {
      const C* tab = p->mixed ? (const C*)p->tsqz32 : (const C*)p->tsqz;
      with_square_side(p->sqz, [&](auto side) {
        constexpr int S = decltype(side)::value;
        const int per_block = kSqWarps * SqLane<S>::G;
        k_zinv_sq<C, S><<<(ny * K1 + per_block - 1) / per_block, kSqWarps * 32, zinv_sq_smem<C, S>(), s>>>(
            g, tab, src, inter);
      });
      JSD_LAUNCHED("k_zinv_sq");
    } else {
      k_zinv<C><<<dim3(K1, ny), 256, sm, s>>>(g, p->fz, twz, src, inter);
      JSD_LAUNCHED("k_zinv");
    }
  }
  {
    ProfScope ps(p, JSD_PROF_XMID, sizeof(C) * (double)(kZinvLines * nsets + 3) * ny * K1 * g.pz, s);
    int rc = launch_xmid<C>(p, p->xmid_variant, inter, out3, s);
    if (rc) return rc;
  }
  {
    const size_t sm = sizeof(C) * ((size_t)g.pz + 6 * (size_t)fline(g.pz));
    ProfScope ps(p, JSD_PROF_ZFWD, sizeof(C) * 3.0 * ny * K1 * g.pz + sizeof(double2) * 3.0 * fs, s);
    if (p->sqz) {
      const C* tab = p->mixed ? (const C*)p->tsqz32 : (const C*)p->tsqz;
      with_square_side(p->sqz, [&](auto side) {
        constexpr int S = decltype(side)::value;
        const int per_block = kSqWarps * SqLane<S>::G;
        k_zfwd_sq<C, S><<<(ny * K1 + per_block - 1) / per_block, kSqWarps * 32, zfwd_sq_smem<C, S>(), s>>>(
            g, tab, out3, p->q, p->H1, p->hg, conv);
      });
      JSD_LAUNCHED("k_zfwd_sq");
    } else {
      k_zfwd<C><<<dim3(K1, ny), 128, sm, s>>>(g, p->fz, twz, out3, p->q, p->H1, p->hg, conv);
      JSD_LAUNCHED("k_zfwd");
    }
  }
  return 0;
}

int stage(jsd_plan* p, double2* state, double* dpdx, int st, int time_step, cudaStream_t s) {
  const Geo& g = p->g;
  const Geo gp = planes_of(g);
  const size_t fs = (size_t)gp.ny * g.nk;
  const int ny = g.ny, ni = g.ny - 2;
  double2* u = state;
  double2* v = state + fs;
  double2* w = state + 2 * fs;
  const double2* uhist = nullptr;
  if (p->desc.kind == JSD_KIND_DUAL && !p->desc.linearise) {
    if (!p->history) return fail(JSD_ERR_STATE, "dual step needs jsd_set_history first");
    const int idx = p->n_history - 1 - time_step;
    if (idx < 0) return fail(JSD_ERR_ARG, "dual time step beyond the registered forward history");
    uhist = p->history + (size_t)idx * 3 * fs;
  }
  int rc = nonlinear(p, state, uhist, st, s);
  if (rc) return rc;
  const int blk = 256;
  if (!p->coupling && p->desc.kind != JSD_KIND_NS) {
    if (p->desc.kind == JSD_KIND_PERTURBATION)
      k_coupling_off<kPerturbation><<<grid_for(fs, blk), blk, 0, s>>>(gp, v, p->dub, p->H1, p->hg);
    else
      k_coupling_off<kDual><<<grid_for(fs, blk), blk, 0, s>>>(gp, u, p->dub, p->H1, p->hg);
    JSD_LAUNCHED("k_coupling_off");
  }
  if (p->src_hv) {
    k_add_source<<<grid_for(fs, blk), blk, 0, s>>>(gp, p->src_hv, p->src_hg, p->src_00, p->H1, p->hg,
                                                   p->conv + (size_t)st * 2 * gp.ny);
    JSD_LAUNCHED("k_add_source");
  }
  if (!p->om_valid) {
    k_omega<<<grid_for(fs, blk), blk, 0, s>>>(gp, u, w, p->om);
    JSD_LAUNCHED("k_omega");
  }
  // eigenbasis transforms. In the mixed form the nonlinear terms q, H1, h_g
  // are FP32-accurate (FP32 transforms and products), so their products run
  // in split TF32 like the y-derivatives and are kept in FP32 (X1, T_0, T_1
  // and the previous stage's terms); V^-1 v and V^-1 omega_y of the state
  // (first stage of a call) stay FP64-accurate. The linearised terms are
  // formed in FP64 and keep FP64-accurate products.
  const bool split_in = p->split_eig_in && !(p->desc.linearise && p->desc.kind != JSD_KIND_NS);
  {
    GemmBatch b = gemm_batch(p);
    const size_t E = p->edoubles;
    const size_t rowd = 2 * (size_t)g.nk * g.nb;  // doubles per Chebyshev row
    if (split_in) {
      rc = launch_split_eig_in(p, s);
      if (rc) return rc;
    } else {
      add_entry(b, p->VinvD, (const double*)p->q, p->X1, ni, ny);
      add_entry(b, p->Vinv, (const double*)p->H1 + rowd, p->T + 0 * E, ni, ni);
      add_entry(b, p->Vinv, (const double*)p->hg + rowd, p->T + 1 * E, ni, ni);
    }
    if (!p->ev_valid) add_entry(b, p->Vinv, (const double*)v + rowd, p->T + 2 * E, ni, ni);
    if (!p->om_valid) add_entry(b, p->Vinv, (const double*)p->om + rowd, p->T + 3 * E, ni, ni);
    if (b.count) {
      rc = launch_eig(p, b, ni, kSiteEigIn, s);
      if (rc) return rc;
    }
  }
  if (p->src_hv) {
    if (split_in)
      k_add_source00<float><<<1, 128, 0, s>>>(g, p->Vinv, p->lda, p->src_hv, reinterpret_cast<float*>(p->X1));
    else
      k_add_source00<double><<<1, 128, 0, s>>>(g, p->Vinv, p->lda, p->src_hv, p->X1);
    JSD_LAUNCHED("k_add_source00");
  }
  {
    EigTables t{p->lam, p->c0, p->cN, p->sgn, p->w0, p->wN, p->re_run};
    StageCoef sc{kAlpha[st], kBeta[st], kGamma[st], kXi[st], p->desc.dt, p->desc.dt_explicit, p->desc.re_tau,
                 st == 0 ? 1 : 0};
    const int N = 2 * g.nk * g.nb;
    const size_t E = p->edoubles;
    // reads X1, 4 transformed fields, 2 old terms; writes 2 old terms, v~, om~
    // (X1, T_0, T_1 and the old terms in FP32 when split)
    ProfScope ps(p, JSD_PROF_EIGEN, sizeof(double) * (split_in ? 7.5 : 11.0) * (double)E, s);
    // v~ and om~ carried from the last stage are read from vnt / omnt and the
    // update goes to their ping-pong partners, which then become vnt / omnt
    const double* vt = p->ev_valid ? p->vnt : p->T + 2 * E;
    const double* omt = p->om_valid ? p->omnt : p->T + 3 * E;
    if (p->ev_valid) std::swap(p->vnt, p->vnt_alt);
    if (p->om_valid) std::swap(p->omnt, p->omnt_alt);
    const int blocks = (N + kEigCols - 1) / kEigCols, rpp = eigen_update_rpp(ny);
    const size_t sm = eigen_update_smem(ny);
    if (split_in)
      k_eigen_update<float><<<blocks, kEigCols * kEigParts, sm, s>>>(
          g, t, sc, reinterpret_cast<const float*>(p->X1), reinterpret_cast<const float*>(p->T),
          reinterpret_cast<const float*>(p->T + E), vt, omt, (const double*)v, reinterpret_cast<float*>(p->hv_old),
          reinterpret_cast<float*>(p->hg_old), p->vnt, p->omnt, rpp);
    else
      k_eigen_update<double><<<blocks, kEigCols * kEigParts, sm, s>>>(
          g, t, sc, p->X1, p->T, p->T + E, vt, omt, (const double*)v, p->hv_old, p->hg_old, p->vnt, p->omnt, rpp);
    JSD_LAUNCHED("k_eigen_update");
  }
  {
    const size_t n2 = 2 * (size_t)ny;
    const double* lns = p->lhs_inv_ns + (size_t)st * n2 * n2;
    const double2* conv = p->conv + (size_t)st * 2 * gp.ny;
    const double2* conv_old = st == 0 ? nullptr : p->conv + (size_t)(st - 1) * 2 * gp.ny;
    const double dte = p->desc.dt_explicit;
    // per-run matrices: lr / lns point at run 0's stage-st matrices, the kernel offsets by run
    const double* lr = p->lr_ns + (size_t)st * n2 * n2;
    const dim3 grid((unsigned)((n2 + kMeanFlowRows - 1) / kMeanFlowRows), (unsigned)g.nb);
    k_mean_flow_rows<<<grid, 32 * kMeanFlowRows, sizeof(double2) * 2 * n2, s>>>(
        g, lr, lns, u, w, conv, conv_old, dpdx, p->dpdx_scale, dte * kGamma[st], dte * kXi[st], p->uw00);
    JSD_LAUNCHED("k_mean_flow_rows");
  }
  {
    GemmBatch b = gemm_batch(p);
    add_entry(b, p->Vfull, p->vnt, (double*)v, ny, ni);
    add_entry(b, p->DVfull, p->vnt, (double*)p->dvn, ny, ni);
    add_entry(b, p->Vfull, p->omnt, (double*)p->om, ny, ni);
    rc = launch_eig(p, b, ny, kSiteEigOut, s);
    if (rc) return rc;
  }
  k_reconstruct<<<grid_for(fs, blk), blk, 0, s>>>(g, p->dvn, p->om, p->uw00, u, v, w, p->errflag);
  JSD_LAUNCHED("k_reconstruct");
  // the back-transform left V^-1 v, V^-1 omega_y and dv/dy of the new state
  p->ev_valid = p->om_valid = p->dv_valid = true;
  return 0;
}

int mass_flux(jsd_plan* p, double2* state, double* dpdx, cudaStream_t s) {
  const Geo& g = p->g;
  const size_t fs = (size_t)g.ny * g.nk;
  k_plane_sums_sliced<<<dim3(g.ny, kSumSlices), 256, 0, s>>>(g, state, 1, 1, p->partial);
  JSD_LAUNCHED("k_plane_sums_sliced");
  k_mass_flux_scalar_sliced<<<1, 32, 0, s>>>(g.ny, p->yw, p->partial, g.c_inv, p->desc.flow_rate_target,
                                             p->desc.dt_explicit, dpdx, p->scal);
  JSD_LAUNCHED("k_mass_flux_scalar_sliced");
  k_roundtrip_shift<<<grid_for(fs, 256), 256, 0, s>>>(g, state, p->scal, p->tmp);
  JSD_LAUNCHED("k_roundtrip_shift");
  JSD_CUDA(cudaMemcpyAsync(state, p->tmp, fs * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  p->om_valid = false;  // u changed; v (and so V^-1 v, dv/dy) did not
  return 0;
}

// Transpose of one stage of the linearised perturbation step (jsd_adjoint.cuh):
// lam holds the cotangent of the stage's output state on entry and of its
// input state on return. hv_old / hg_old carry the cotangents of the terms a
// stage hands to the next (`last`: none, for the last stage of a step);
// adj_conv[st] the cotangent of the stage's conv00.
int stage_adj(jsd_plan* p, double2* lam, int st, bool last, cudaStream_t s) {
  const Geo& g = p->g;
  const size_t fs = (size_t)g.ny * g.nk;
  const int ny = g.ny, ni = g.ny - 2;
  const size_t E = p->edoubles;
  const size_t rowd = 2 * (size_t)g.nk;
  double2 *lu = lam, *lv = lam + fs, *lw = lam + 2 * fs;
  const int blk = 256;
  // 9'
  k_reconstruct_adj<<<grid_for(fs, blk), blk, 0, s>>>(g, lu, lw, p->dvn, p->om, p->adj_ub);
  JSD_LAUNCHED("k_reconstruct_adj");
  // 8': cotangents of V^-1 v (from v and from dv/dy) and of V^-1 omega_y
  {
    GemmBatch b = gemm_batch(p);
    add_entry(b, p->Vfull_T, (const double*)lv, p->T + 0 * E, ni, ny);
    add_entry(b, p->DVfull_T, (const double*)p->dvn, p->T + 1 * E, ni, ny);
    add_entry(b, p->Vfull_T, (const double*)p->om, p->T + 2 * E, ni, ny);
    int rc = launch_gemm(p, b, ni, kSiteEigIn, s);
    if (rc) return rc;
  }
  // 6'
  {
    EigTables t{p->lam, p->c0, p->cN, p->sgn, p->w0, p->wN, nullptr};
    StageCoef sc{kAlpha[st], kBeta[st], kGamma[st], kXi[st], p->desc.dt, p->desc.dt_explicit, p->desc.re_tau,
                 st == 0 ? 1 : 0};
    const int N = 2 * g.nk;
    k_eigen_update_adj<<<(N + kEigCols - 1) / kEigCols, kEigCols * kEigParts, 0, s>>>(
        g, t, sc, last ? 1 : 0, p->T + 0 * E, p->T + 1 * E, p->T + 2 * E, p->hv_old, p->hg_old, p->X1, p->T + 3 * E,
        p->vnt, p->omnt, p->vnt_alt, (double*)p->tmp);
    JSD_LAUNCHED("k_eigen_update_adj");
  }
  // 7'
  {
    const size_t n2 = 2 * (size_t)ny;
    const double dte = p->desc.dt_explicit;
    const unsigned grid = (unsigned)((n2 + kMeanFlowRows - 1) / kMeanFlowRows);
    k_mean_flow_adj<<<grid, 32 * kMeanFlowRows, 0, s>>>(g, p->lr_T + (size_t)st * n2 * n2, p->li_T + (size_t)st * n2 * n2,
                                                        p->adj_ub, dte * kGamma[st], dte * kXi[st], p->adj_x00,
                                                        p->adj_conv + (size_t)st * n2,
                                                        st > 0 ? p->adj_conv + (size_t)(st - 1) * n2 : nullptr);
    JSD_LAUNCHED("k_mean_flow_adj");
  }
  // 5': cotangents of q (all rows), H1, h_g, the interior of v and of omega_y
  {
    GemmBatch b = gemm_batch(p);
    add_entry(b, p->VinvD_T, p->X1, (double*)p->q, ny, ni);
    add_entry(b, p->Vinv_T, p->T + 3 * E, (double*)p->H1 + rowd, ni, ni);
    add_entry(b, p->Vinv_T, p->vnt, (double*)p->hg + rowd, ni, ni);
    add_entry(b, p->Vinv_T, p->omnt, (double*)p->tmp + rowd, ni, ni);
    add_entry(b, p->Vinv_T, p->vnt_alt, (double*)p->Dfld + rowd, ni, ni);
    int rc = launch_gemm(p, b, ny, kSiteEigOut, s);
    if (rc) return rc;
  }
  // 4' .. 2': the state cotangent but D^T dv_bar, and dv_bar
  {
    const size_t n2 = 2 * (size_t)ny;
    k_linear_terms_adj<<<grid_for(fs, blk), blk, 0, s>>>(g, p->ub, p->dub, p->q, p->H1, p->hg,
                                                        p->adj_conv + (size_t)st * n2, p->Dfld, p->tmp, p->adj_x00,
                                                        lu, lv, lw, p->Dfld + fs);
    JSD_LAUNCHED("k_linear_terms_adj");
  }
  // 1': v_bar += D^T dv_bar
  {
    GemmBatch b = gemm_batch(p);
    add_entry(b, p->D_T, (const double*)(p->Dfld + fs), (double*)(p->Dfld + 2 * fs), ny, ny);
    int rc = launch_gemm(p, b, ny, kSiteDfield, s);
    if (rc) return rc;
  }
  k_add_field<<<grid_for(fs, blk), blk, 0, s>>>(fs, p->Dfld + 2 * fs, lv);
  JSD_LAUNCHED("k_add_field");
  return 0;
}

int set_smem_limits() {
  static bool done = false;
  if (done) return 0;
  const int big = 200 * 1024;
  JSD_CUDA(cudaFuncSetAttribute(k_zinv<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_zinv<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_xmid<double2, kXmidZB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_xmid<float2, kXmidZB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_xmid_dual<double2, kXmidZB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_xmid_dual<float2, kXmidZB>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_zfwd<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_zfwd<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_sgemm3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sgemm3Smem::BYTES));
  for (int c = 0; c < kDgemmConfigs; ++c) {
    cudaError_t e = cudaSuccess;
    with_dgemm_cfg(c, [&](auto cfg) {
      using Cfg = decltype(cfg);
      e = cudaFuncSetAttribute(k_dgemm_t<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::BYTES);
    });
    JSD_CUDA(e);
  }
  JSD_CUDA(cudaFuncSetAttribute(k_mean_flow, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_mean_flow_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_eigen_update<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_eigen_update<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  JSD_CUDA(cudaFuncSetAttribute(k_tc05_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
  JSD_CUDA(cudaFuncSetAttribute(k_oz8_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kOzSmem));
  cudaError_t err = cudaSuccess;
  for (int sd : kSquareSides)
    with_square_side(sd, [&](auto side) {
      constexpr int S = decltype(side)::value;
      const void* fns[] = {(const void*)k_zinv_sq<double2, S>,      (const void*)k_zinv_sq<float2, S>,
                           (const void*)k_zfwd_sq<double2, S>,      (const void*)k_zfwd_sq<float2, S>,
                           (const void*)k_xmid_sq<double2, S>,      (const void*)k_xmid_sq<float2, S>,
                           (const void*)k_xmid_dual_sq<double2, S>, (const void*)k_xmid_dual_sq<float2, S>};
      if constexpr (S % 2 == 0) {
        for (const void* fn : {(const void*)k_xmid_h2<double2, S>, (const void*)k_xmid_h2<float2, S>}) {
          const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
          if (e != cudaSuccess) err = e;
        }
      }
      for (const void* fn : fns) {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        if (e != cudaSuccess) err = e;
      }
    });
  JSD_CUDA(err);
  done = true;
  return 0;
}

void destroy(jsd_plan* p) {
  if (!p) return;
  for (auto& r : p->recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : p->ev_free) cudaEventDestroy(e);
  for (void* a : p->allocs) cudaFree(a);
  delete p;
}

// ---------------------------------------------------------------------------
// Allocation-free energy reduction. Its only scratch (one partial sum per
// y-plane) is this file-scope device array: every GPU that loads the library
// holds it until the process exits. In host code `g_static_partial` is a
// host-side stand-in, not a device address; the device address is looked up
// with cudaGetSymbolAddress once per device (with that device current) and
// cached.
// ---------------------------------------------------------------------------
constexpr int kStaticMaxNy = 4096;
static __device__ __align__(256) double g_static_partial[kStaticMaxNy];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mutex;
double* g_static_partial_addr[kStaticMaxDevices] = {nullptr};

int static_partial_address(double** out) {
  int dev = -1;
  JSD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticMaxDevices) return fail(JSD_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_partial_addr[dev]) {
    void* ptr = nullptr;
    JSD_CUDA(cudaGetSymbolAddress(&ptr, g_static_partial));
    g_static_partial_addr[dev] = static_cast<double*>(ptr);
  }
  *out = g_static_partial_addr[dev];
  return 0;
}

}  // namespace

extern "C" {

int jsd_energy_noalloc(const void* state, int mx, int ny, int mz, int px_ref, int pz_ref, double lx, double lz,
                       const double* y_weights, double* out, void* stream) {
  if (!state || !y_weights || !out) return fail(JSD_ERR_ARG, "null argument");
  if (mx < 1 || mz < 1 || (mx % 2) == 0 || (mz % 2) == 0 || ny < 2 || px_ref < 1 || pz_ref < 1 || lx <= 0 ||
      lz <= 0)
    return fail(JSD_ERR_ARG, "invalid grid");
  if (ny > kStaticMaxNy)
    return fail(JSD_ERR_ARG, "jsd_energy_noalloc supports at most " + std::to_string(kStaticMaxNy) +
                                 " Chebyshev points (got " + std::to_string(ny) + ")");
  double* partial = nullptr;
  int rc = static_partial_address(&partial);
  if (rc) return rc;
  Geo g{};
  g.mx = mx;
  g.ny = ny;
  g.mz = mz;
  g.kx_max = mx / 2;
  g.kz_max = mz / 2;
  g.nk = mx * mz;
  g.nb = 1;
  const double two_pi = 2.0 * M_PI;
  const double s = (lx / two_pi) * (lz / two_pi);
  g.c_inv = s / std::sqrt((double)px_ref * (double)pz_ref);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // k_plane_sums overwrites partial[0 .. ny) before k_weighted_total reads it,
  // so nothing left by an earlier call is used
  k_plane_sums<<<ny, 256, 0, st>>>(g, static_cast<const double2*>(state), 3, 0, partial);
  JSD_LAUNCHED("k_plane_sums");
  k_weighted_total<<<1, 32, 0, st>>>(ny, y_weights, partial, 0.25 * g.c_inv * g.c_inv, out);
  JSD_LAUNCHED("k_weighted_total");
  return 0;
}

int jsd_abi_version(void) { return JSD_ABI_VERSION; }

int jsd_profile_enable(jsd_plan* plan, int enable) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  plan->profiling = enable != 0;
  return 0;
}

int jsd_profile_read(jsd_plan* plan, int kernel_class, double* total_ms, long long* launches, double* work) {
  if (!plan || !total_ms || !launches || !work) return fail(JSD_ERR_ARG, "null argument");
  double ms = 0, w = 0;
  long long n = 0;
  std::vector<jsd_plan::Rec> keep;
  for (auto& r : plan->recs) {
    if (r.cls != kernel_class) {
      keep.push_back(r);
      continue;
    }
    float t = 0;
    JSD_CUDA(cudaEventSynchronize(r.b));
    JSD_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
    ms += t;
    w += r.work;
    ++n;
    plan->ev_free.push_back(r.a);
    plan->ev_free.push_back(r.b);
  }
  plan->recs.swap(keep);
  *total_ms = ms;
  *launches = n;
  *work = w;
  return 0;
}

const char* jsd_last_error(void) { return g_last_error.c_str(); }

size_t jsd_workspace_bytes(const jsd_plan* plan) { return plan ? plan->ws_bytes : 0; }

int jsd_autotune(jsd_plan* plan, void* stream) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo& g = plan->g;
  const int ny = g.ny, ni = g.ny - 2;
  const size_t fs = (size_t)ny * g.nk * g.nb;
  const size_t E = plan->edoubles;
  const size_t rowd = 2 * (size_t)g.nk * g.nb;
  // the timed products read these workspace fields: give them defined values
  for (double2* f : {plan->q, plan->H1, plan->hg})
    JSD_CUDA(cudaMemsetAsync(f, 0, fs * sizeof(double2), s));
  for (double* f : {plan->vnt, plan->omnt}) JSD_CUDA(cudaMemsetAsync(f, 0, E * sizeof(double), s));
  cudaEvent_t e0, e1;
  JSD_CUDA(cudaEventCreate(&e0));
  JSD_CUDA(cudaEventCreate(&e1));
  int rc = 0;
  for (int site = 0; site < kGemmSites && rc == 0; ++site) {
    if (site == kSiteDfield && plan->mixed) continue;  // the mixed form's y-derivatives run k_sgemm3
    GemmBatch b = gemm_batch(plan);
    int max_m = ny;
    if (site == kSiteDfield) {
      // steady-state stage: D on u and w
      add_entry(b, plan->Dm, (const double*)plan->q, (double*)plan->Dfld, ny, ny);
      add_entry(b, plan->Dm, (const double*)plan->H1, (double*)(plan->Dfld + 2 * fs), ny, ny);
    } else if (site == kSiteEigIn) {
      const bool linear = plan->desc.linearise && plan->desc.kind != JSD_KIND_NS;
      if (plan->split_eig_in && !linear) {
        // the nonlinear terms go to the split kernel: what stays on this site
        // is V^-1 omega_y at the first stage after a mass-flux correction
        add_entry(b, plan->Vinv, (const double*)plan->H1 + rowd, plan->T + 3 * E, ni, ni);
      } else {
        add_entry(b, plan->VinvD, (const double*)plan->q, plan->X1, ni, ny);
        add_entry(b, plan->Vinv, (const double*)plan->H1 + rowd, plan->T, ni, ni);
        add_entry(b, plan->Vinv, (const double*)plan->hg + rowd, plan->T + E, ni, ni);
      }
      max_m = ni;
    } else {
      add_entry(b, plan->Vfull, plan->vnt, (double*)plan->tmp, ny, ni);
      add_entry(b, plan->DVfull, plan->vnt, (double*)plan->dvn, ny, ni);
      add_entry(b, plan->Vfull, plan->omnt, (double*)plan->om, ny, ni);
    }
    float best = 3.0e38f;
    for (int c = 0; c < kDgemmConfigs && rc == 0; ++c) {
      rc = launch_gemm_cfg(plan, b, max_m, c, s);  // warm-up
      if (rc) break;
      if (cudaEventRecord(e0, s) != cudaSuccess) rc = fail(JSD_ERR_CUDA, "cudaEventRecord");
      for (int r = 0; r < 5 && rc == 0; ++r) rc = launch_gemm_cfg(plan, b, max_m, c, s);
      if (rc) break;
      float ms = 0.f;
      if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = fail(JSD_ERR_CUDA, "autotune timing");
        break;
      }
      plan->tune_ms[site][c] = ms / 5.f;
      if (ms < best) {
        best = ms;
        plan->gemm_cfg[site] = c;
      }
    }
    // eigenbasis sites of mixed plans: the Ozaki int8 kernel against the best DMMA tile
    if (rc == 0 && site != kSiteDfield && plan->oz_ready && plan->mixed) {
      plan->eig_ms[site][0] = best / 5.f;
      rc = launch_ozaki(plan, b, s);  // warm-up
      if (rc == 0 && cudaEventRecord(e0, s) != cudaSuccess) rc = fail(JSD_ERR_CUDA, "cudaEventRecord");
      for (int r = 0; r < 5 && rc == 0; ++r) rc = launch_ozaki(plan, b, s);
      float ms = 0.f;
      if (rc == 0 && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                      cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        rc = fail(JSD_ERR_CUDA, "autotune timing");
      if (rc == 0) {
        plan->eig_ms[site][1] = ms / 5.f;
        plan->eig_kernel[site] = ms < best ? 1 : 0;
      }
    }
  }
  // split-TF32 product kernels (mixed plans)
  if (rc == 0 && plan->mixed && plan->tc_rows) {
    const double* src[2] = {(const double*)plan->q, (const double*)plan->H1};
    double* dst[2] = {(double*)plan->Dfld, (double*)(plan->Dfld + 2 * fs)};
    float best = 3.0e38f;
    // both calls of a steady stage that use the kernel: D on u and w, and
    // the split eigenbasis-in products when the plan splits them
    const int keep = plan->split_kernel;
    auto run = [&](int k) {
      int r = launch_dfield(plan, src, dst, 2, s, true, k);
      if (r == 0 && plan->split_eig_in) {
        plan->split_kernel = k;
        r = launch_split_eig_in(plan, s);
        plan->split_kernel = keep;
      }
      return r;
    };
    for (int k = 0; k < 2 && rc == 0; ++k) {
      rc = run(k);  // warm-up
      if (rc) break;
      if (cudaEventRecord(e0, s) != cudaSuccess) rc = fail(JSD_ERR_CUDA, "cudaEventRecord");
      for (int r = 0; r < 5 && rc == 0; ++r) rc = run(k);
      if (rc) break;
      float ms = 0.f;
      if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = fail(JSD_ERR_CUDA, "autotune timing");
        break;
      }
      plan->split_ms[k] = ms / 5.f;
      if (ms < best) {
        best = ms;
        plan->split_kernel = k;
      }
    }
  }
  // x-pass kernel variants (nonlinear plans)
  const bool linear = plan->desc.linearise && plan->desc.kind != JSD_KIND_NS;
  if (rc == 0 && !linear) {
    float best = 3.0e38f;
    for (int v = 0; v < 3 && rc == 0; ++v) {
      if (!xmid_available(plan, v)) continue;
      auto run = [&]() {
        return plan->mixed ? launch_xmid<float2>(plan, v, (float2*)plan->inter, (float2*)plan->out3, s)
                           : launch_xmid<double2>(plan, v, (double2*)plan->inter, (double2*)plan->out3, s);
      };
      rc = run();  // warm-up
      if (rc) break;
      if (cudaEventRecord(e0, s) != cudaSuccess) rc = fail(JSD_ERR_CUDA, "cudaEventRecord");
      for (int r = 0; r < 3 && rc == 0; ++r) rc = run();
      if (rc) break;
      float ms = 0.f;
      if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        rc = fail(JSD_ERR_CUDA, "autotune timing");
        break;
      }
      plan->xmid_ms[v] = ms / 3.f;
      if (ms < best) {
        best = ms;
        plan->xmid_variant = v;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int jsd_split_kernel(const jsd_plan* plan, float* times_ms) {
  if (!plan) return -1;
  if (times_ms)
    for (int k = 0; k < 2; ++k) times_ms[k] = plan->split_ms[k];
  return plan->mixed ? plan->split_kernel : -1;
}

int jsd_set_split_kernel(jsd_plan* plan, int kernel) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if (!plan->mixed || kernel < 0 || kernel > 1 || (kernel == 1 && !plan->tc_rows))
    return fail(JSD_ERR_ARG, "split-TF32 kernel not available for this plan");
  plan->split_kernel = kernel;
  return 0;
}

int jsd_split_eig_in(const jsd_plan* plan) {
  if (!plan) return -1;
  return plan->mixed ? (plan->split_eig_in ? 1 : 0) : -1;
}

int jsd_set_split_eig_in(jsd_plan* plan, int on) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if (!plan->mixed || !plan->ei_hi[0] || (on != 0 && on != 1))
    return fail(JSD_ERR_ARG, "split eigenbasis-in products need a mixed-precision plan (Ny - 2 <= 144)");
  plan->split_eig_in = on == 1;
  return 0;
}

int jsd_eig_kernel(const jsd_plan* plan, int site, float* times_ms) {
  if (!plan || (site != kSiteEigIn && site != kSiteEigOut)) return -1;
  if (times_ms)
    for (int k = 0; k < 2; ++k) times_ms[k] = plan->eig_ms[site][k];
  return plan->oz_ready ? plan->eig_kernel[site] : 0;
}

int jsd_set_eig_kernel(jsd_plan* plan, int site, int kernel) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if ((site != kSiteEigIn && site != kSiteEigOut) || kernel < 0 || kernel > 1 || (kernel == 1 && !plan->oz_ready))
    return fail(JSD_ERR_ARG, "eigenbasis kernel not available for this plan and site");
  plan->eig_kernel[site] = kernel;
  return 0;
}

int jsd_device_error(jsd_plan* plan, void* stream) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  int h = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  JSD_CUDA(cudaMemcpyAsync(&h, plan->errflag, sizeof(int), cudaMemcpyDeviceToHost, s));
  JSD_CUDA(cudaStreamSynchronize(s));
  if (h) {
    JSD_CUDA(cudaMemsetAsync(plan->errflag, 0, sizeof(int), s));
    JSD_CUDA(cudaStreamSynchronize(s));
    if (h & kErrWaitExpired)
      return fail(JSD_ERR_CUDA, "a kernel's bounded wait expired (tcgen05 accumulator or bulk copy did not complete)");
    return fail(JSD_ERR_NONFINITE, "the state became non-finite (NaN or infinity after a stage)");
  }
  return 0;
}

int jsd_set_wait_limit(jsd_plan* plan, int polls) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if (polls < 0) return fail(JSD_ERR_ARG, "wait limit must be >= 0 (0 restores the default)");
  plan->wait_limit = polls == 0 ? kWaitPolls : polls;
  return 0;
}

int jsd_wait_limit(const jsd_plan* plan) { return plan ? plan->wait_limit : 0; }

int jsd_xmid_variant(const jsd_plan* plan, float* times_ms) {
  if (!plan) return -1;
  if (times_ms)
    for (int v = 0; v < 3; ++v) times_ms[v] = plan->xmid_ms[v];
  return plan->xmid_variant;
}

int jsd_set_xmid_variant(jsd_plan* plan, int variant) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if (variant < 0 || variant > 2 || !xmid_available(plan, variant))
    return fail(JSD_ERR_ARG, "x-pass variant not available for this plan");
  plan->xmid_variant = variant;
  return 0;
}

int jsd_set_gemm_config(jsd_plan* plan, int site, int config) {
  if (!plan || site < 0 || site >= kGemmSites || config < 0 || config >= kDgemmConfigs)
    return fail(JSD_ERR_ARG, "bad GEMM site or configuration");
  plan->gemm_cfg[site] = config;
  return 0;
}

int jsd_gemm_config(const jsd_plan* plan, int site, float* times_ms) {
  if (!plan || site < 0 || site >= kGemmSites) return -1;
  if (times_ms)
    for (int c = 0; c < kDgemmConfigs; ++c) times_ms[c] = plan->tune_ms[site][c];
  return plan->gemm_cfg[site];
}

int jsd_launches_first_step_extra(const jsd_plan* plan) {
  if (!plan) return 0;
  const bool linear = plan->desc.linearise && plan->desc.kind != JSD_KIND_NS;
  // the first stage of a call derives omega_y (k_omega) and, for the linear
  // terms, dv/dy (one GEMM) from the caller's state
  const bool cmf = plan->desc.constant_mass_flux != 0;
  return (cmf ? 0 : 1) + (linear ? 1 : 0);
}

int jsd_launches_per_step(const jsd_plan* plan) {
  if (!plan) return 0;
  const bool linear = plan->desc.linearise && plan->desc.kind != JSD_KIND_NS;
  // steady state: each stage launches dfield (not for the linear terms, which take
  // dv/dy carried from the last stage), nonlinear terms (3 transforms or 1 linear
  // kernel), 2 GEMMs, eigen update, mean flow and reconstruct; omega_y is carried
  // too, except after the mass-flux correction (3 launches) changed u
  const bool coupling_off = !plan->coupling && plan->desc.kind != JSD_KIND_NS;
  // a source (jsd_set_source) adds k_add_source and k_add_source00 per stage
  const int per_stage = (linear ? 6 : 9) + (coupling_off ? 1 : 0) + (plan->src_hv ? 2 : 0);
  const bool cmf = plan->desc.constant_mass_flux != 0;
  return 3 * per_stage + (cmf ? 3 + 1 : 0);
}

int jsd_plan_create(const jsd_desc* d, jsd_plan** out) {
  if (!d || !out) return fail(JSD_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->mx < 3 || d->mz < 3 || (d->mx % 2) == 0 || (d->mz % 2) == 0)
    return fail(JSD_ERR_ARG, "mx and mz must be odd and >= 3");
  if (d->ny < 4) return fail(JSD_ERR_ARG, "ny must be >= 4");
  if (d->kind < 0 || d->kind > 2) return fail(JSD_ERR_ARG, "unknown equation kind");
  if (!d->D || !d->V || !d->Vinv || !d->lam || !d->sgn || !d->c0 || !d->cN || !d->w0 || !d->wN ||
      !d->y_weights || !d->rhs_ns || !d->lhs_inv_ns)
    return fail(JSD_ERR_ARG, "operator tables missing");
  if (d->kind != JSD_KIND_NS && (!d->base_u || !d->base_du))
    return fail(JSD_ERR_ARG, "perturbation and dual equations need the base profile");
  if (d->re_tau == 0.0 || d->dt == 0.0 || d->dt_explicit == 0.0) return fail(JSD_ERR_ARG, "zero Re or dt");
  const int nb = d->n_batch > 1 ? d->n_batch : 1;
  if (nb > 1) {
    if (d->kind == JSD_KIND_DUAL || d->constant_mass_flux)
      return fail(JSD_ERR_ARG, "batches of runs support the NS and perturbation equations without mass-flux control");
    if (!d->re_tau_batch) return fail(JSD_ERR_ARG, "a batch needs re_tau_batch");
    for (int r = 0; r < nb; ++r)
      if (d->re_tau_batch[r] == 0.0) return fail(JSD_ERR_ARG, "zero Re in re_tau_batch");
  }
  int rc = set_smem_limits();
  if (rc) return rc;

  jsd_plan* p = new jsd_plan();
  p->desc = *d;
  p->mixed = d->precision == JSD_PRECISION_MIXED;
  Geo& g = p->g;
  g.mx = d->mx;
  g.ny = d->ny;
  g.mz = d->mz;
  g.kx_max = d->mx / 2;
  g.kz_max = d->mz / 2;
  g.px = d->px_fft > 0 ? d->px_fft : choose_fft_size(d->mx);
  g.pz = d->pz_fft > 0 ? d->pz_fft : choose_fft_size(d->mz);
  g.nk = d->mx * d->mz;
  g.nb = nb;
  p->nb_max = nb;
  const double two_pi = 2.0 * M_PI;
  g.ax = two_pi / d->lx;
  g.az = two_pi / d->lz;
  const double s = (d->lx / two_pi) * (d->lz / two_pi);
  g.c_inv = s / std::sqrt((double)d->px_ref * (double)d->pz_ref);
  g.c_fwd = std::sqrt((double)d->px_ref * (double)d->pz_ref) / (s * (double)g.px * (double)g.pz);
  p->dpdx_scale = std::sqrt(((double)d->px_ref * (two_pi / d->lx) * (two_pi / d->lx)) *
                            ((double)d->pz_ref * (two_pi / d->lz) * (two_pi / d->lz)));
  if (!square_side(g.px) && (size_t)kXmidZB * g.px > (size_t)kXmidEPT * kXmidThreads) {
    destroy(p);
    return fail(JSD_ERR_ARG, "x FFT length too large for the x-pass kernel (max " +
                                 std::to_string(kXmidEPT * kXmidThreads / kXmidZB) + ")");
  }
  if (g.px < 3 * g.kx_max + 1 || g.pz < 3 * g.kz_max + 1) {
    destroy(p);
    return fail(JSD_ERR_ARG, "FFT length below 3K+1 would alias the quadratic products");
  }
  std::vector<double2> twx, twz;
  if (!build_fft(g.px, p->fx, twx) || !build_fft(g.pz, p->fz, twz)) {
    destroy(p);
    return fail(JSD_ERR_ARG, "FFT length must factor into 2, 3, 5, 7");
  }
  const int ny = d->ny, ni = ny - 2;
  p->lda = (ny + 15) / 16 * 16;
  p->fdoubles = 2 * (size_t)ny * g.nk * nb;
  p->edoubles = 2 * (size_t)ni * g.nk * nb;
  const size_t fs = (size_t)ny * g.nk * nb;  // complex entries per field (all runs)
  const size_t n2 = 2 * (size_t)ny;

  std::vector<double> VinvD((size_t)ni * ny, 0.0), Vfull((size_t)ny * ni, 0.0), DVfull((size_t)ny * ni, 0.0);
  for (int i = 0; i < ni; ++i)
    for (int c = 0; c < ny; ++c) {
      long double acc = 0;
      for (int j = 0; j < ni; ++j) acc += (long double)d->Vinv[(size_t)i * ni + j] * d->D[(size_t)(j + 1) * ny + c];
      VinvD[(size_t)i * ny + c] = (double)acc;
    }
  for (int r = 0; r < ni; ++r)
    for (int c = 0; c < ni; ++c) Vfull[(size_t)(r + 1) * ni + c] = d->V[(size_t)r * ni + c];
  for (int r = 0; r < ny; ++r)
    for (int c = 0; c < ni; ++c) {
      long double acc = 0;
      for (int j = 0; j < ni; ++j) acc += (long double)d->D[(size_t)r * ny + j + 1] * d->V[(size_t)j * ni + c];
      DVfull[(size_t)r * ni + c] = (double)acc;
    }

#define JSD_TRY(x)        \
  do {                    \
    int rc_ = (x);        \
    if (rc_) {            \
      destroy(p);         \
      return rc_;         \
    }                     \
  } while (0)

  JSD_TRY(upload(p, &p->twx, twx.data(), twx.size()));
  JSD_TRY(upload(p, &p->twz, twz.data(), twz.size()));
  p->sqx = square_side(g.px);
  p->sqz = square_side(g.pz);
  p->xmid_variant = default_xmid_variant(p);
  // default tiles before any autotuning: the two-stage 48- or 64-row tile that
  // pads the call site's row count least (configurations 0 and 1)
  for (int site = 0; site < kGemmSites; ++site) {
    const int m = site == kSiteEigIn ? ny - 2 : ny;
    p->gemm_cfg[site] = ((m + 47) / 48 * 48 < (m + 63) / 64 * 64) ? 0 : 1;
  }
  for (int axis = 0; axis < 2; ++axis) {
    const int n = axis == 0 ? g.px : g.pz;
    if (!(axis == 0 ? p->sqx : p->sqz)) continue;
    std::vector<double2> tab(n);
    std::vector<float2> tab32(n);
    for (int e = 0; e < n; ++e) {
      const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)n;
      tab[e] = make_double2((double)cosl(ang), (double)sinl(ang));
      tab32[e] = make_float2((float)tab[e].x, (float)tab[e].y);
    }
    JSD_TRY(upload(p, axis == 0 ? &p->tsqx : &p->tsqz, tab.data(), tab.size()));
    JSD_TRY(upload(p, axis == 0 ? &p->tsqx32 : &p->tsqz32, tab32.data(), tab32.size()));
  }
  if (p->mixed) {
    std::vector<float2> tx(twx.size()), tz(twz.size());
    for (size_t i = 0; i < twx.size(); ++i) tx[i] = make_float2((float)twx[i].x, (float)twx[i].y);
    for (size_t i = 0; i < twz.size(); ++i) tz[i] = make_float2((float)twz[i].x, (float)twz[i].y);
    JSD_TRY(upload(p, &p->twx32, tx.data(), tx.size()));
    JSD_TRY(upload(p, &p->twz32, tz.data(), tz.size()));
    // D = D_hi + D_lo with both parts representable in TF32 (round to nearest)
    std::vector<float> hi((size_t)ny * p->lda, 0.f), lo((size_t)ny * p->lda, 0.f);
    for (int r = 0; r < ny; ++r)
      for (int c = 0; c < ny; ++c) {
        const double x = d->D[(size_t)r * ny + c];
        const float h = tf32_round((float)x);
        hi[(size_t)r * p->lda + c] = h;
        lo[(size_t)r * p->lda + c] = tf32_round((float)(x - (double)h));
      }
    JSD_TRY(upload(p, &p->Dhi, hi.data(), hi.size()));
    JSD_TRY(upload(p, &p->Dlo, lo.data(), lo.size()));
    // V^-1 D and V^-1 split the same way (eigenbasis-in products of the
    // FP32-accurate nonlinear terms)
    const double* eiA[2] = {VinvD.data(), d->Vinv};
    const int eiK[2] = {ny, ni};
    for (int k = 0; k < 2; ++k) {
      std::vector<float> eh((size_t)ni * p->lda, 0.f), el((size_t)ni * p->lda, 0.f);
      for (int r = 0; r < ni; ++r)
        for (int c = 0; c < eiK[k]; ++c) {
          const double x = eiA[k][(size_t)r * eiK[k] + c];
          const float h = tf32_round((float)x);
          eh[(size_t)r * p->lda + c] = h;
          el[(size_t)r * p->lda + c] = tf32_round((float)(x - (double)h));
        }
      JSD_TRY(upload(p, &p->ei_hi[k], eh.data(), eh.size()));
      JSD_TRY(upload(p, &p->ei_lo[k], el.data(), el.size()));
    }
    // on by default for the Navier-Stokes equations; with a base flow
    // (perturbation, dual) its coupling terms are part of these products, and
    // over 2000 steps at 48 x 65 x 48 splitting them raised the mixed form's
    // energy-history error against FP64 from 2e-7 to 1.2e-6, so such plans
    // keep FP64-accurate products unless asked (jsd_set_split_eig_in)
    p->split_eig_in = ni <= Sgemm3Smem::BM && d->kind == JSD_KIND_NS;
    if (ny <= kTcM + 1) {
      p->tc_rows = ny;
      std::vector<float> ahi, alo;
      tc05_pack_a(d->D, ny, ny, ny, tf32_round, ahi, alo);
      JSD_TRY(upload(p, &p->tc_ahi, ahi.data(), ahi.size()));
      JSD_TRY(upload(p, &p->tc_alo, alo.data(), alo.size()));
      for (int k = 0; k < 2; ++k) {
        tc05_pack_a(eiA[k], ni, eiK[k], eiK[k], tf32_round, ahi, alo);
        JSD_TRY(upload(p, &p->tc_ei_hi[k], ahi.data(), ahi.size()));
        JSD_TRY(upload(p, &p->tc_ei_lo[k], alo.data(), alo.size()));
      }
      if (ny > kTcM) {
        std::vector<double> xr(kTcKp, 0.0);
        for (int c = 0; c < ny; ++c) xr[c] = d->D[(size_t)kTcM * ny + c];
        JSD_TRY(upload(p, &p->tc_xrow, xr.data(), xr.size()));
      }
      // the tcgen05 kernel is the default (58 us per call against 86 us for
      // k_sgemm3 at 128 x 129 x 128); the autotuner re-decides per plan
      p->split_kernel = 1;
    }
  }
  JSD_TRY(dev_alloc(p, (void**)&p->errflag, sizeof(int)));
  JSD_CUDA(cudaMemset(p->errflag, 0, sizeof(int)));
  {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
      p->num_sms = sms;
  }
  JSD_TRY(upload_padded(p, &p->Dm, d->D, ny, ny, p->lda));
  JSD_TRY(upload_padded(p, &p->VinvD, VinvD.data(), ni, ny, p->lda));
  JSD_TRY(upload_padded(p, &p->Vinv, d->Vinv, ni, ni, p->lda));
  JSD_TRY(upload_padded(p, &p->Vfull, Vfull.data(), ny, ni, p->lda));
  JSD_TRY(upload_padded(p, &p->DVfull, DVfull.data(), ny, ni, p->lda));
  if (ny <= kOzM + 1) {
    // int8 slice packs of the four eigenbasis operators (V^-1 D: K = Ny; V and
    // D V: M = Ny; at most one of M, K above 128). FP64 plans may select the
    // kernel too (jsd_set_eig_kernel); only the mixed form's autotuning does.
    const double* hostA[4] = {VinvD.data(), d->Vinv, Vfull.data(), DVfull.data()};
    const int Ms[4] = {ni, ni, ny, ny}, Ks[4] = {ny, ni, ni, ni};
    const double* devA[4] = {p->VinvD, p->Vinv, p->Vfull, p->DVfull};
    for (int k = 0; k < 4; ++k) {
      OzPackA pk;
      oz_pack_a(hostA[k], Ms[k], Ks[k], Ks[k], pk);
      JSD_TRY(upload(p, &p->oz_a[k], pk.slices.data(), pk.slices.size()));
      JSD_TRY(upload(p, &p->oz_rs[k], pk.row_scale.data(), pk.row_scale.size()));
      JSD_TRY(upload(p, &p->oz_xr[k], pk.xrow.data(), pk.xrow.size()));
      JSD_TRY(upload(p, &p->oz_xc[k], pk.xcol.data(), pk.xcol.size()));
      p->oz_src[k] = devA[k];
    }
    // (the epilogue's pair stores need 16-byte aligned rows: every output is a
    // double2 field or an even offset into one, with an even row stride 2 nk nb)
    p->oz_ready = tensor_map_encoder() != nullptr;
    // the mixed form starts on the int8 kernel at both eigenbasis sites (the
    // autotuner keeps whichever is faster per site); FP64 plans on DMMA
    if (p->oz_ready && p->mixed) p->eig_kernel[kSiteEigIn] = p->eig_kernel[kSiteEigOut] = 1;
  }
  {
    // small boxes: with fewer than 8 tiles of 32 columns per SM in a two-field
    // call the persistent tcgen05 pipelines never fill (their operand loads
    // and set-up dominate), so such plans start on k_sgemm3 and DMMA
    const long long tiles = 2 * ((2LL * g.nk * nb + 31) / 32);
    if (tiles < 8LL * p->num_sms) {
      p->split_kernel = 0;
      p->eig_kernel[kSiteEigIn] = p->eig_kernel[kSiteEigOut] = 0;
    }
  }
  JSD_TRY(upload(p, &p->lam, d->lam, ni));
  JSD_TRY(upload(p, &p->sgn, d->sgn, ni));
  JSD_TRY(upload(p, &p->c0, d->c0, ni));
  JSD_TRY(upload(p, &p->cN, d->cN, ni));
  JSD_TRY(upload(p, &p->w0, d->w0, ni));
  JSD_TRY(upload(p, &p->wN, d->wN, ni));
  JSD_TRY(upload(p, &p->yw, d->y_weights, ny));
  JSD_TRY(upload(p, &p->rhs_ns, d->rhs_ns, (size_t)nb * 3 * n2 * n2));
  JSD_TRY(upload(p, &p->lhs_inv_ns, d->lhs_inv_ns, (size_t)nb * 3 * n2 * n2));
  if (nb > 1) JSD_TRY(upload(p, &p->re_run, d->re_tau_batch, (size_t)nb));
  {
    // LR = Linv_ns R_ns for every run and stage (the matrices are block
    // structured, so zero entries of Linv are skipped)
    std::vector<double> lr((size_t)nb * 3 * n2 * n2);
    for (size_t m = 0; m < (size_t)nb * 3; ++m) {
      const double* L = d->lhs_inv_ns + m * n2 * n2;
      const double* R = d->rhs_ns + m * n2 * n2;
      double* O = lr.data() + m * n2 * n2;
      for (size_t i = 0; i < n2; ++i) {
        double* row = O + i * n2;
        std::fill(row, row + n2, 0.0);
        for (size_t k = 0; k < n2; ++k) {
          const double lik = L[i * n2 + k];
          if (lik == 0.0) continue;
          const double* rk = R + k * n2;
          for (size_t j = 0; j < n2; ++j) row[j] += lik * rk[j];
        }
      }
    }
    JSD_TRY(upload(p, &p->lr_ns, lr.data(), lr.size()));
    if (d->kind == JSD_KIND_PERTURBATION && d->linearise && nb == 1 && !d->constant_mass_flux) {
      // transposes for the discrete adjoint (jsd_step_adjoint)
      std::vector<double> lrT(lr.size()), liT(lr.size());
      for (size_t m = 0; m < 3; ++m)
        for (size_t i = 0; i < n2; ++i)
          for (size_t j = 0; j < n2; ++j) {
            lrT[m * n2 * n2 + j * n2 + i] = lr[m * n2 * n2 + i * n2 + j];
            liT[m * n2 * n2 + j * n2 + i] = d->lhs_inv_ns[m * n2 * n2 + i * n2 + j];
          }
      JSD_TRY(upload(p, &p->lr_T, lrT.data(), lrT.size()));
      JSD_TRY(upload(p, &p->li_T, liT.data(), liT.size()));
      auto transpose = [](const double* a, int rows, int cols) {
        std::vector<double> t((size_t)rows * cols);
        for (int r = 0; r < rows; ++r)
          for (int c = 0; c < cols; ++c) t[(size_t)c * rows + r] = a[(size_t)r * cols + c];
        return t;
      };
      const std::vector<double> vdT = transpose(VinvD.data(), ni, ny), viT = transpose(d->Vinv, ni, ni),
                                vfT = transpose(Vfull.data(), ny, ni), dvT = transpose(DVfull.data(), ny, ni),
                                dT = transpose(d->D, ny, ny);
      JSD_TRY(upload_padded(p, &p->VinvD_T, vdT.data(), ny, ni, p->lda));
      JSD_TRY(upload_padded(p, &p->Vinv_T, viT.data(), ni, ni, p->lda));
      JSD_TRY(upload_padded(p, &p->Vfull_T, vfT.data(), ni, ny, p->lda));
      JSD_TRY(upload_padded(p, &p->DVfull_T, dvT.data(), ni, ny, p->lda));
      JSD_TRY(upload_padded(p, &p->D_T, dT.data(), ny, ny, p->lda));
      JSD_TRY(dev_alloc(p, (void**)&p->adj_conv, 3 * n2 * sizeof(double2)));
      JSD_TRY(dev_alloc(p, (void**)&p->adj_x00, n2 * sizeof(double2)));
      JSD_TRY(dev_alloc(p, (void**)&p->adj_ub, n2 * sizeof(double2)));
    }
  }
  if (d->base_u) JSD_TRY(upload(p, &p->ub, d->base_u, ny));
  if (d->base_du) JSD_TRY(upload(p, &p->dub, d->base_du, ny));

  const bool linear = d->linearise && d->kind != JSD_KIND_NS;
  const size_t K1 = g.kx_max + 1;
  const int nsets = (d->kind == JSD_KIND_DUAL) ? 2 : 1;
  JSD_TRY(dev_alloc(p, (void**)&p->Dfld, 3 * (size_t)nsets * fs * sizeof(double2)));
  if (!linear) {
    const size_t csz = p->mixed ? sizeof(float2) : sizeof(double2);
    JSD_TRY(dev_alloc(p, (void**)&p->inter, (size_t)kZinvLines * nsets * ny * nb * K1 * g.pz * csz));
    JSD_TRY(dev_alloc(p, (void**)&p->out3, 3 * (size_t)ny * nb * K1 * g.pz * csz));
  }
  for (double2** f : {&p->q, &p->H1, &p->hg, &p->om, &p->dvn, &p->tmp})
    JSD_TRY(dev_alloc(p, (void**)f, fs * sizeof(double2)));
  JSD_TRY(dev_alloc(p, (void**)&p->conv, 3 * n2 * nb * sizeof(double2)));
  JSD_TRY(dev_alloc(p, (void**)&p->uw00, n2 * nb * sizeof(double2)));
  JSD_TRY(dev_alloc(p, (void**)&p->X1, p->edoubles * sizeof(double)));
  JSD_TRY(dev_alloc(p, (void**)&p->T, 4 * p->edoubles * sizeof(double)));
  for (double** f : {&p->hv_old, &p->hg_old, &p->vnt, &p->omnt, &p->vnt_alt, &p->omnt_alt})
    JSD_TRY(dev_alloc(p, (void**)f, p->edoubles * sizeof(double)));
  JSD_TRY(dev_alloc(p, (void**)&p->partial, (size_t)ny * nb * kSumSlices * sizeof(double)));
  JSD_TRY(dev_alloc(p, (void**)&p->scal, 8 * sizeof(double)));
  // conv entries are only written at (0,0); clear once so every read is defined
  JSD_CUDA(cudaMemset(p->conv, 0, 3 * n2 * nb * sizeof(double2)));
#undef JSD_TRY
  *out = p;
  return 0;
}

int jsd_plan_destroy(jsd_plan* plan) {
  destroy(plan);
  return 0;
}

int jsd_set_source(jsd_plan* plan, const void* hv, const void* hg, const void* s00) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  const bool any = hv || hg || s00, all = hv && hg && s00;
  if (any && !all) return fail(JSD_ERR_ARG, "source terms: give all three arrays or none");
  if (any && plan->g.nb != 1) return fail(JSD_ERR_ARG, "source terms need a single-run plan");
  plan->src_hv = static_cast<const double2*>(hv);
  plan->src_hg = static_cast<const double2*>(hg);
  plan->src_00 = static_cast<const double2*>(s00);
  return 0;
}

int jsd_set_history(jsd_plan* plan, const void* states, int n_states) {
  if (!plan || (!states && n_states > 0) || n_states < 0) return fail(JSD_ERR_ARG, "bad history");
  plan->history = static_cast<const double2*>(states);
  plan->n_history = n_states;
  return 0;
}

// n_steps full steps; uses (and refreshes) the carried eigen-space state
int run_steps(jsd_plan* plan, double2* st, double* dpdx, int first_step, int n_steps, cudaStream_t s) {
  for (int t = 0; t < n_steps; ++t) {
    for (int k = 0; k < 3; ++k) {
      int rc = stage(plan, st, dpdx, k, first_step + t, s);
      if (rc) return rc;
    }
    if (plan->desc.constant_mass_flux) {
      int rc = mass_flux(plan, st, dpdx, s);
      if (rc) return rc;
    }
  }
  return 0;
}

int jsd_step(jsd_plan* plan, void* state, double* dpdx, int first_step, int n_steps, void* stream) {
  if (!plan || !state || !dpdx || n_steps < 0) return fail(JSD_ERR_ARG, "null argument");
  plan->ev_valid = plan->om_valid = plan->dv_valid = false;  // the caller may have changed the state
  return run_steps(plan, static_cast<double2*>(state), dpdx, first_step, n_steps, static_cast<cudaStream_t>(stream));
}

int jsd_step_trajectory(jsd_plan* plan, void* state, double* dpdx, int first_step, int n_steps, void* states,
                        void* stream) {
  if (!plan || !state || !dpdx || !states || n_steps < 0) return fail(JSD_ERR_ARG, "null argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = 3 * (size_t)plan->g.ny * plan->g.nk * plan->g.nb * sizeof(double2);
  char* out = static_cast<char*>(states);
  JSD_CUDA(cudaMemcpyAsync(out, state, bytes, cudaMemcpyDeviceToDevice, s));
  plan->ev_valid = plan->om_valid = plan->dv_valid = false;
  for (int t = 0; t < n_steps; ++t) {
    int rc = run_steps(plan, static_cast<double2*>(state), dpdx, first_step + t, 1, s);
    if (rc) return rc;
    JSD_CUDA(cudaMemcpyAsync(out + (size_t)(t + 1) * bytes, state, bytes, cudaMemcpyDeviceToDevice, s));
  }
  return 0;
}

int jsd_correct_mass_flux(jsd_plan* plan, void* state, double* dpdx, void* stream) {
  if (!plan || !state) return fail(JSD_ERR_ARG, "null argument");
  if (plan->g.nb > 1) return fail(JSD_ERR_ARG, "single-run entry point called on a batch plan (see jsd_energy_runs)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* dp = dpdx ? dpdx : plan->scal + 1;  // a scratch slot when the caller keeps no pressure gradient
  plan->ev_valid = plan->om_valid = plan->dv_valid = false;
  return mass_flux(plan, static_cast<double2*>(state), dp, s);
}

int jsd_energy(jsd_plan* plan, const void* state, double* out, void* stream) {
  if (!plan || !state || !out) return fail(JSD_ERR_ARG, "null argument");
  if (plan->g.nb > 1) return fail(JSD_ERR_ARG, "single-run entry point called on a batch plan (see jsd_energy_runs)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo& g = plan->g;
  k_plane_sums_sliced<<<dim3(g.ny, kSumSlices), 256, 0, s>>>(g, static_cast<const double2*>(state), 3, 0,
                                                              plan->partial);
  JSD_LAUNCHED("k_plane_sums_sliced");
  k_weighted_total_sliced<<<1, 32, 0, s>>>(g.ny, plan->yw, plan->partial, 0.25 * g.c_inv * g.c_inv, out);
  JSD_LAUNCHED("k_weighted_total_sliced");
  return 0;
}

int jsd_energy_runs(jsd_plan* plan, const void* state, double* out, void* stream) {
  if (!plan || !state || !out) return fail(JSD_ERR_ARG, "null argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo& g = plan->g;
  const Geo gp = planes_of(g);
  k_plane_sums_sliced<<<dim3(gp.ny, kSumSlices), 256, 0, s>>>(gp, static_cast<const double2*>(state), 3, 0,
                                                               plan->partial);
  JSD_LAUNCHED("k_plane_sums_sliced");
  k_weighted_total_runs_sliced<<<g.nb, 32, 0, s>>>(g.ny, g.nb, plan->yw, plan->partial, 0.25 * g.c_inv * g.c_inv,
                                                    out);
  JSD_LAUNCHED("k_weighted_total_runs_sliced");
  return 0;
}

int jsd_step_adjoint(jsd_plan* plan, void* cotangent, int n_steps, void* stream) {
  if (!plan || !cotangent || n_steps < 0) return fail(JSD_ERR_ARG, "null argument");
  if (!plan->VinvD_T)
    return fail(JSD_ERR_ARG, "the discrete adjoint covers linearised perturbation plans of one run without "
                             "mass-flux control");
  if (!plan->coupling) return fail(JSD_ERR_ARG, "the discrete adjoint needs coupling_term on");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n2 = 2 * (size_t)plan->g.ny;
  double2* lam = static_cast<double2*>(cotangent);
  for (int t = 0; t < n_steps; ++t) {
    JSD_CUDA(cudaMemsetAsync(plan->adj_conv, 0, 3 * n2 * sizeof(double2), s));
    for (int st = 2; st >= 0; --st) {
      int rc = stage_adj(plan, lam, st, st == 2, s);
      if (rc) return rc;
    }
  }
  // the workspace the forward step carries between stages was overwritten
  plan->ev_valid = plan->om_valid = plan->dv_valid = false;
  return 0;
}

int jsd_energy_grad(jsd_plan* plan, const void* state, void* out, void* stream) {
  if (!plan || !state || !out) return fail(JSD_ERR_ARG, "null argument");
  if (plan->g.nb > 1) return fail(JSD_ERR_ARG, "single-run entry point called on a batch plan (see jsd_energy_runs)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo& g = plan->g;
  const size_t total = 3 * (size_t)g.ny * g.nk;
  k_energy_grad<<<grid_for(total, 256), 256, 0, s>>>(g, static_cast<const double2*>(state), plan->yw,
                                                    0.5 * g.c_inv * g.c_inv, static_cast<double2*>(out));
  JSD_LAUNCHED("k_energy_grad");
  return 0;
}

int jsd_set_coupling_term(jsd_plan* plan, int on) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if (plan->desc.kind == JSD_KIND_NS && !on) return fail(JSD_ERR_ARG, "coupling_term applies to perturbation equations");
  plan->coupling = on != 0;
  return 0;
}

int jsd_set_base_flow(jsd_plan* plan, const double* base_u, const double* base_du, void* stream) {
  if (!plan || !base_u || !base_du) return fail(JSD_ERR_ARG, "null argument");
  if (!plan->ub || !plan->dub) return fail(JSD_ERR_STATE, "the plan has no base flow");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = (size_t)plan->g.ny * sizeof(double);
  JSD_CUDA(cudaMemcpyAsync(plan->ub, base_u, bytes, cudaMemcpyDeviceToDevice, s));
  JSD_CUDA(cudaMemcpyAsync(plan->dub, base_du, bytes, cudaMemcpyDeviceToDevice, s));
  return 0;
}

int jsd_set_batch_active(jsd_plan* plan, int n_runs) {
  if (!plan) return fail(JSD_ERR_ARG, "null plan");
  if (n_runs < 1 || n_runs > plan->nb_max) return fail(JSD_ERR_ARG, "active runs must be in [1, n_batch]");
  plan->g.nb = n_runs;
  plan->ev_valid = plan->om_valid = plan->dv_valid = false;
  return 0;
}

int jsd_batch_active(const jsd_plan* plan) { return plan ? plan->g.nb : 0; }

int jsd_flow_rate(jsd_plan* plan, const void* u_field, double* out, void* stream) {
  if (!plan || !u_field || !out) return fail(JSD_ERR_ARG, "null argument");
  if (plan->g.nb > 1) return fail(JSD_ERR_ARG, "single-run entry point called on a batch plan (see jsd_energy_runs)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo& g = plan->g;
  k_plane_sums_sliced<<<dim3(g.ny, kSumSlices), 256, 0, s>>>(g, static_cast<const double2*>(u_field), 1, 1,
                                                              plan->partial);
  JSD_LAUNCHED("k_plane_sums_sliced");
  k_weighted_total_sliced<<<1, 32, 0, s>>>(g.ny, plan->yw, plan->partial, g.c_inv, out);
  JSD_LAUNCHED("k_weighted_total_sliced");
  return 0;
}

int jsd_nonlinear_terms(jsd_plan* plan, const void* state, int time_step, void* h_v, void* h_g, void* stream) {
  if (!plan || !state || !h_v || !h_g) return fail(JSD_ERR_ARG, "null argument");
  if (plan->g.nb > 1) return fail(JSD_ERR_ARG, "single-run entry point called on a batch plan (see jsd_energy_runs)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Geo& g = plan->g;
  const size_t fs = (size_t)g.ny * g.nk;
  const double2* uhist = nullptr;
  if (plan->desc.kind == JSD_KIND_DUAL && !plan->desc.linearise) {
    if (!plan->history) return fail(JSD_ERR_STATE, "dual step needs jsd_set_history first");
    const int idx = plan->n_history - 1 - time_step;
    if (idx < 0) return fail(JSD_ERR_ARG, "time step beyond the registered forward history");
    uhist = plan->history + (size_t)idx * 3 * fs;
  }
  plan->ev_valid = plan->om_valid = plan->dv_valid = false;
  int rc = nonlinear(plan, static_cast<const double2*>(state), uhist, 0, s);
  if (rc) return rc;
  GemmBatch b = gemm_batch(plan);
  add_entry(b, plan->Dm, (const double*)plan->q, (double*)plan->tmp, g.ny, g.ny);
  rc = launch_gemm(plan, b, g.ny, kSiteEigIn, s);
  if (rc) return rc;
  k_assemble_hv<<<grid_for(fs, 256), 256, 0, s>>>(g, plan->tmp, plan->H1, static_cast<double2*>(h_v));
  JSD_LAUNCHED("k_assemble_hv");
  JSD_CUDA(cudaMemcpyAsync(h_g, plan->hg, fs * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  return 0;
}

}  // extern "C"
