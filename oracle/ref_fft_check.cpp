// Test infrastructure: checks the oracle's FFT substitute (ref_support/fft_substitute.cpp) against a
// naive O(N^2) DFT, for the layouts the reference's own FFT tests cover (tests/test_fft.cpp:118-240):
// both signs, strided and batched 1D, 2D with interleaved batches, scale applied only to the
// transformed elements (padding untouched), real-to-complex and complex-to-real. Prints the worst
// relative error per case and exits non-zero if any exceeds 1e-13.
#include <cmath>
#include <complex>
#include <cstdio>
#include <numbers>
#include <vector>

#include "fft/fftw_fft.hpp"

using cplx = std::complex<double>;
using namespace spodvr;

namespace {
std::vector<cplx> random_values(std::size_t n, unsigned seed) {
  std::vector<cplx> v(n);
  std::uint64_t x = seed;
  for (auto& c : v) {
    x = x * 6364136223846793005ULL + 1442695040888963407ULL;
    const double re = double(x >> 11) / double(1ULL << 53) - 0.5;
    x = x * 6364136223846793005ULL + 1442695040888963407ULL;
    c = {re, double(x >> 11) / double(1ULL << 53) - 0.5};
  }
  return v;
}

void naive_line(std::vector<cplx>& a, std::size_t off, int n, int stride, double sign) {
  std::vector<long double> re(n), im(n);
  for (int k = 0; k < n; ++k) {
    long double sr = 0, si = 0;
    for (int j = 0; j < n; ++j) {
      const long double ang = sign * 2.0L * std::numbers::pi_v<long double> * ((long(j) * k) % n) / n;
      const cplx x = a[off + std::size_t(j) * stride];
      sr += x.real() * std::cos(ang) - x.imag() * std::sin(ang);
      si += x.real() * std::sin(ang) + x.imag() * std::cos(ang);
    }
    re[k] = sr;
    im[k] = si;
  }
  for (int k = 0; k < n; ++k) a[off + std::size_t(k) * stride] = cplx(double(re[k]), double(im[k]));
}

double rel_err(const std::vector<cplx>& a, const std::vector<cplx>& b) {
  double d = 0, s = 0;
  for (std::size_t i = 0; i < a.size(); ++i) {
    d = std::max(d, std::abs(a[i] - b[i]));
    s = std::max(s, std::abs(b[i]));
  }
  return d / s;
}

int failures = 0;
void report(const char* name, int n, double err) {
  const bool ok = err <= 1e-13;
  if (!ok) ++failures;
  std::printf("%-28s n=%-5d rel_err=%.3e %s\n", name, n, err, ok ? "ok" : "FAIL");
}
}  // namespace

int main() {
  const FftwFft fft;
  const int lengths[] = {2, 4, 6, 8, 10, 12, 16, 18, 20, 22, 28, 30, 32, 36, 40, 44, 48, 56, 60, 64, 70, 88, 96, 110,
                         128, 154, 176, 180, 240, 256, 280, 384, 512, 97};
  for (const int n : lengths) {
    for (const FftSign sign : {FftSign::Minus, FftSign::Plus}) {
      const double s = sign == FftSign::Plus ? 1.0 : -1.0;
      // Strided, batched 1D with padding between batches (stride 3, distance 3n + 2).
      const int howmany = 3, stride = 3, dist = 3 * n + 2;
      std::vector<cplx> a = random_values(std::size_t(dist) * howmany, 7 + n);
      std::vector<cplx> ref = a;
      fft.plan_complex({n, howmany, stride, dist}, sign, 0.5)->execute(a);
      for (int b = 0; b < howmany; ++b) {
        naive_line(ref, std::size_t(b) * dist, n, stride, s);
        for (int i = 0; i < n; ++i) ref[std::size_t(b) * dist + std::size_t(i) * stride] *= 0.5;
      }
      report(sign == FftSign::Plus ? "1d strided batched (+)" : "1d strided batched (-)", n, rel_err(a, ref));
    }
  }
  // 2D with interleaved batches: element (o, i) of batch b at b + o*(ni*hb) + i*hb.
  const int pairs[][2] = {{8, 4}, {64, 32}, {176, 56}, {16, 16}, {280, 56}, {12, 10}};
  for (const auto& pr : pairs) {
    const int no = pr[0], ni = pr[1], hb = 3;
    std::vector<cplx> a = random_values(std::size_t(no) * ni * hb, 11);
    std::vector<cplx> ref = a;
    fft.plan_complex_2d({no, ni * hb, ni, hb, hb, 1}, FftSign::Minus, 0.25)->execute(a);
    for (int b = 0; b < hb; ++b) {
      for (int o = 0; o < no; ++o) naive_line(ref, b + std::size_t(o) * ni * hb, ni, hb, -1.0);
      for (int i = 0; i < ni; ++i) naive_line(ref, b + std::size_t(i) * hb, no, ni * hb, -1.0);
    }
    for (auto& v : ref) v *= 0.25;
    report("2d interleaved (-)", no * ni, rel_err(a, ref));
  }
  // Real to complex and back (sign +, scale 1; then sign -, scale 1/n): the identity.
  for (const int n : {8, 12, 56, 96, 110}) {
    std::vector<double> x(n);
    for (int i = 0; i < n; ++i) x[i] = std::sin(0.3 * i) + 0.1 * i;
    std::vector<cplx> half(n / 2 + 1);
    fft.plan_real_to_complex({n}, {n / 2 + 1}, FftSign::Plus, 1.0)->execute(x, half);
    std::vector<cplx> full(n);
    for (int i = 0; i < n; ++i) full[i] = x[i];
    naive_line(full, 0, n, 1, 1.0);
    std::vector<cplx> head(full.begin(), full.begin() + n / 2 + 1);
    report("r2c (+)", n, rel_err(half, head));
    std::vector<double> back(n);
    fft.plan_complex_to_real({n / 2 + 1}, {n}, FftSign::Minus, 1.0 / n)->execute(half, back);
    double d = 0;
    for (int i = 0; i < n; ++i) d = std::max(d, std::abs(back[i] - x[i]));
    report("c2r (-) round trip", n, d);
  }
  std::printf("%s\n", failures == 0 ? "ALL OK" : "FAILURES");
  return failures == 0 ? 0 : 1;
}
