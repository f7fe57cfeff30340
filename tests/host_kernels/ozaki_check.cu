// Host-side check of the Ozaki int8 product (jsd_ozaki.cuh): packs A with
// oz_pack_a and 32-column tiles of B the way the converter warps do (balanced
// digits of oz_pack_b; slices
// stacked into one 256-row operand), emulates the tensor-core products by
// reading both operands back through their canonical-layout offsets (int32
// accumulation per diagonal), combines like
// the epilogue (FP64 extras for row 128 / column 128 included) and compares
// with a long-double product. Prints per case: M K error/(|A||B|) max,
// relative Frobenius error, and the same two for a plain FP64 product.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../jax-spectral-dns_b200/csrc/jsd_ozaki.cuh"

using namespace jsd;

static double urand(unsigned long long& s) {
  s = s * 6364136223846793005ull + 1442695040888963407ull;
  return ((s >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
}

static void run_case(int M, int K, int N, unsigned long long seed) {
  std::vector<double> A((size_t)M * K), B((size_t)K * N);
  // rows and columns with different magnitudes (and one zero column)
  for (int i = 0; i < M; ++i)
    for (int k = 0; k < K; ++k) A[(size_t)i * K + k] = urand(seed) * std::pow(10.0, 3.0 * urand(seed)) / (1 + i);
  for (int k = 0; k < K; ++k)
    for (int j = 0; j < N; ++j)
      B[(size_t)k * N + j] = j == 5 ? 0.0 : urand(seed) * std::exp(-k / 20.0) * std::pow(10.0, 4.0 * urand(seed));
  OzPackA pa;
  oz_pack_a(A.data(), M, K, K, pa);
  const int kt = K < kOzK ? K : kOzK, mt = M < kOzM ? M : kOzM;
  std::vector<double> C((size_t)M * N, 0.0);
  std::vector<unsigned char> bs(kOzBBytes);
  for (int n0 = 0; n0 < N; n0 += kOzN) {
    double colscale[kOzN], bx[kOzN], xdot[kOzN];
    for (int lane = 0; lane < kOzN; ++lane) {
      const int col = n0 + lane;
      double v[kOzK];
      double mx = 0.0;
      for (int k = 0; k < kOzK; ++k) {
        v[k] = (col < N && k < kt) ? B[(size_t)k * N + col] : 0.0;
        mx = std::fmax(mx, std::fabs(v[k]));
      }
      bx[lane] = (K > kOzK && col < N) ? B[(size_t)kOzK * N + col] : 0.0;
      double dot = 0.0;
      if (M > kOzM) {  // converter warps of kOzConvRows rows each, partials summed in warp order
        for (int w = 0; w < kOzConvWarps; ++w) {
          double part = 0.0;
          for (int j = 0; j < kOzConvRows; ++j)
            if (kOzConvRows * w + j < kt) part = std::fma(pa.xrow[kOzConvRows * w + j], v[kOzConvRows * w + j], part);
          dot = w == 0 ? part : dot + part;
        }
      }
      xdot[lane] = dot;
      const int eb = oz_exponent(mx);
      colscale[lane] = oz_pow2(eb + 2);
      const double sc = oz_pow2(54 - eb);
      for (int k0 = 0; k0 < kOzK; k0 += 16) {
        double xs[16];
        for (int j = 0; j < 16; ++j) xs[j] = v[k0 + j] * sc;
        uint32_t w[kOzSlices][4];
        oz_pack_b<4>(xs, w);
        for (int q = 0; q < kOzSlices; ++q)
          for (int j = 0; j < 16; ++j)
            bs[oz_offset(kOzBRows, q * kOzN + lane, k0) + j] = (unsigned char)((w[q][j >> 2] >> (8 * (j & 3))) & 0xFFu);
      }
    }
    for (int r = 0; r < mt; ++r)
      for (int lane = 0; lane < kOzN && n0 + lane < N; ++lane) {
        long long acc[kOzDiags] = {};
        for (int d = 0; d < kOzDiags; ++d)
          for (int p = 1; p <= kOzSlices; ++p) {
            const int q = d + 2 - p;
            if (q < 1 || q > kOzSlices) continue;
            long long s = 0;
            for (int k = 0; k < kOzK; ++k)
              s += (long long)pa.slices[(size_t)(p - 1) * kOzASlice + oz_offset(kOzM, r, k)] *
                   (long long)(signed char)bs[oz_offset(kOzBRows, (q - 1) * kOzN + lane, k)];
            acc[d] += s;
          }
        for (int d = 0; d < kOzDiags; ++d)
          if (acc[d] >= (1ll << 31) || acc[d] < -(1ll << 31)) std::printf("overflow\n");
        double rr = (double)acc[kOzDiags - 1];
        for (int d = kOzDiags - 2; d >= 0; --d) rr = std::fma(rr, 0.0078125, (double)acc[d]);
        const double xc = K > kOzK ? pa.xcol[r] : 0.0;
        C[(size_t)r * N + n0 + lane] = std::fma(xc, bx[lane], rr * pa.row_scale[r] * colscale[lane]);
      }
    if (M > kOzM)
      for (int lane = 0; lane < kOzN && n0 + lane < N; ++lane) C[(size_t)kOzM * N + n0 + lane] = xdot[lane];
  }
  double emax = 0, e2 = 0, x2 = 0, dmax = 0, d2 = 0;
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      long double ex = 0, sa = 0;
      double dg = 0;
      for (int k = 0; k < K; ++k) {
        ex += (long double)A[(size_t)i * K + k] * B[(size_t)k * N + j];
        sa += std::fabs(A[(size_t)i * K + k] * B[(size_t)k * N + j]);
        dg += A[(size_t)i * K + k] * B[(size_t)k * N + j];
      }
      const double err = (double)std::fabs((long double)C[(size_t)i * N + j] - ex);
      const double derr = (double)std::fabs((long double)dg - ex);
      if (sa > 0) {
        emax = std::fmax(emax, err / (double)sa);
        dmax = std::fmax(dmax, derr / (double)sa);
      }
      e2 += err * err;
      d2 += derr * derr;
      x2 += (double)(ex * ex);
    }
  std::printf("%d %d %.3e %.3e %.3e %.3e\n", M, K, emax, std::sqrt(e2 / x2), dmax, std::sqrt(d2 / x2));
}

int main() {
  run_case(127, 129, 70, 1);   // V^-1 D: K = 129 (column 128 in FP64)
  run_case(127, 127, 64, 2);   // V^-1
  run_case(129, 127, 45, 3);   // V (walls), D V: M = 129 (row 128 in FP64)
  run_case(65, 63, 33, 4);     // a smaller grid
  return 0;
}
