// Host-side check of the register FFT building blocks (jsd_fftsq.cuh): the
// prime-factor S-point DFTs and the two-stage square transform of length S*S,
// with the lanes of a group emulated one after another. Prints, per S and
// direction, the largest error against a direct DFT relative to the largest
// output magnitude.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../jax-spectral-dns_b200/csrc/jsd_fftsq.cuh"

using namespace jsd;

static double urand(unsigned& s) {
  s = s * 1664525u + 1013904223u;
  return ((s >> 8) & 0xffffff) / double(0x1000000) - 0.5;
}

template <int S, bool INV>
static double check_square() {
  constexpr int N = S * S;
  unsigned seed = 12345u + S * 7u + (INV ? 1u : 0u);
  std::vector<double2> x(N), ref(N), out(N);
  for (int i = 0; i < N; ++i) x[i] = make_double2(urand(seed), urand(seed));
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int k = 0; k < N; ++k) {
    long double re = 0, im = 0;
    for (int n = 0; n < N; ++n) {
      const long double a = (INV ? 2 : -2) * pi * (long double)((long long)n * k % N) / N;
      re += x[n].x * cosl(a) - x[n].y * sinl(a);
      im += x[n].x * sinl(a) + x[n].y * cosl(a);
    }
    ref[k] = make_double2((double)re, (double)im);
  }
  std::vector<double2> table(N);
  for (int e = 0; e < N; ++e) {
    const long double a = -2 * pi * e / N;
    table[e] = make_double2((double)cosl(a), (double)sinl(a));
  }
  std::vector<double2> xb(sq_xbuf<S>());
  double2 reg[S][S];
  for (int t = 0; t < S; ++t) {
    double2 tw[S > 1 ? S - 1 : 1];
    sq_twiddles<S>(tw, table.data(), t);
    for (int m = 0; m < S; ++m) reg[t][m] = x[t + S * m];
    sq_stage1<S, INV>(reg[t], tw, xb.data(), t);
  }
  for (int t = 0; t < S; ++t) {
    sq_stage2<S, INV>(reg[t], xb.data(), t);
    for (int m = 0; m < S; ++m) out[t + S * m] = reg[t][m];
  }
  double err = 0, mag = 0;
  for (int k = 0; k < N; ++k) {
    err = fmax(err, fmax(fabs(out[k].x - ref[k].x), fabs(out[k].y - ref[k].y)));
    mag = fmax(mag, fmax(fabs(ref[k].x), fabs(ref[k].y)));
  }
  return err / mag;
}

// the half-split form (even S): lanes (t, h) hold positions t + S (2 j + h)
template <int S, bool INV>
static double check_half() {
  constexpr int N = S * S, H = S / 2;
  unsigned seed = 777u + S * 13u + (INV ? 1u : 0u);
  std::vector<double2> x(N), ref(N), out(N);
  for (int i = 0; i < N; ++i) x[i] = make_double2(urand(seed), urand(seed));
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int k = 0; k < N; ++k) {
    long double re = 0, im = 0;
    for (int n = 0; n < N; ++n) {
      const long double a = (INV ? 2 : -2) * pi * (long double)((long long)n * k % N) / N;
      re += x[n].x * cosl(a) - x[n].y * sinl(a);
      im += x[n].x * sinl(a) + x[n].y * cosl(a);
    }
    ref[k] = make_double2((double)re, (double)im);
  }
  std::vector<double2> table(N);
  for (int e = 0; e < N; ++e) {
    const long double a = -2 * pi * e / N;
    table[e] = make_double2((double)cosl(a), (double)sinl(a));
  }
  std::vector<double2> xb(sq_xbuf<S>());
  double2 reg[S][2][H];
  for (int t = 0; t < S; ++t)
    for (int h = 0; h < 2; ++h) {
      for (int j = 0; j < H; ++j) reg[t][h][j] = x[t + S * (2 * j + h)];
      dft_reg<H, INV>(reg[t][h]);
    }
  for (int t = 0; t < S; ++t)
    for (int h = 0; h < 2; ++h)
      for (int k = 0; k < H; ++k)
        xb[(h * H + k) * (S + 1) + t] =
            sq2_butterfly<S, INV>(reg[t][h][k], reg[t][1 - h][k], k, table.data(), t, h);
  for (int t = 0; t < S; ++t)
    for (int h = 0; h < 2; ++h) {
      sq2_stage2<S, INV>(reg[t][h], xb.data(), table.data(), t, h);
      for (int j = 0; j < H; ++j) out[t + S * (2 * j + h)] = reg[t][h][j];
    }
  double err = 0, mag = 0;
  for (int k = 0; k < N; ++k) {
    err = fmax(err, fmax(fabs(out[k].x - ref[k].x), fabs(out[k].y - ref[k].y)));
    mag = fmax(mag, fmax(fabs(ref[k].x), fabs(ref[k].y)));
  }
  return err / mag;
}

template <int S>
static void half() {
  printf("h%d %.3e %.3e\n", S, check_half<S, false>(), check_half<S, true>());
}

template <int S>
static void both() {
  printf("%d %.3e %.3e\n", S, check_square<S, false>(), check_square<S, true>());
}

int main() {
  both<2>(); both<3>(); both<4>(); both<5>(); both<6>(); both<7>(); both<8>(); both<10>(); both<12>();
  both<14>(); both<15>(); both<20>(); both<21>(); both<24>(); both<28>(); both<30>();
  half<4>(); half<10>(); half<14>(); half<6>(); half<8>();
  return 0;
}
