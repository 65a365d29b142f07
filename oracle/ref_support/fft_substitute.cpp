// Test infrastructure (oracle build only): an FP64 FFT behind the reference's Fft interface.
//
// The reference's CPU path calls its FFT library through spodvr::Fft (src/fft/fft.hpp:12-73); its
// only implementation, FftwFft (src/fft/fftw_fft.cpp), needs FFTW3 or oneMKL, neither of which
// exists on these machines. This file defines FftwFft's four plan factories with a project-written
// mixed-radix Stockham FFT, so that the reference's own sources compile unchanged around it. The
// contract kept from src/fft/fftw_fft.cpp:
//   - sign Minus = exp(-2 pi i k n / N), sign Plus = exp(+...) (fft.hpp:9-11);
//   - in place on the caller's array; element (o, i) of batch b at b*distance + o*os + i*is;
//   - the scale is applied after the transform, only when it differs from 1, and only to the
//     transformed elements (fftw_fft.cpp:60-71, apply_scale);
//   - real-to-complex: the half spectrum; complex-to-real: the imaginary parts of k = 0 and
//     k = N/2 are ignored, the input is not modified (fft.hpp:41-55).
// Accuracy: twiddles from std::cos/std::sin of the reduced angle, O(eps log N) relative error like
// FFTW's; the reference accepts FFT-library differences of this size.
#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <numbers>
#include <stdexcept>
#include <vector>

#include "fft/fftw_fft.hpp"

namespace spodvr {

namespace {

using cplx = std::complex<double>;

// One 1D transform of length n and a fixed sign, as a list of mixed-radix Stockham stages with their
// twiddles precomputed: stage with radix r after sub-transforms of length ns uses w_(ns r)^(t k),
// k < ns, t < r; the small DFTs use the r-th roots of unity.
class Line {
 public:
  Line(int n, FftSign sign) : n_(n), sign_(sign == FftSign::Plus ? 1.0 : -1.0) {
    int m = n;
    std::vector<int> radices;
    while (m % 4 == 0) {
      radices.push_back(4);
      m /= 4;
    }
    for (int p = 2; m > 1; ++p)
      while (m % p == 0) {
        radices.push_back(p);
        m /= p;
      }
    int ns = 1;
    for (const int r : radices) {
      Stage st{r, ns, {}, {}};
      st.twiddle.resize(std::size_t(ns) * r);
      for (int k = 0; k < ns; ++k)
        for (int t = 0; t < r; ++t) st.twiddle[std::size_t(k) * r + t] = root(static_cast<long>(t) * k, ns * r);
      st.roots.resize(r);
      for (int q = 0; q < r; ++q) st.roots[q] = root(q, r);
      stages_.push_back(std::move(st));
      ns *= r;
      r_max_ = std::max(r_max_, r);
    }
  }

  int size() const { return n_; }

  // Transforms x (contiguous, n values); work: n values of scratch. The result ends in x.
  void run(cplx* x, cplx* work) const {
    if (n_ == 1) return;
    cplx* in = x;
    cplx* out = work;
    cplx fixed[128];
    std::vector<cplx> heap;
    if (r_max_ > 64) heap.resize(2 * std::size_t(r_max_));
    cplx* a = r_max_ > 64 ? heap.data() : fixed;
    cplx* b = a + r_max_;
    for (const Stage& st : stages_) {
      const int r = st.radix;
      const int ns = st.ns;
      const int stride = n_ / r;
      const int span = ns * r;
      for (int j0 = 0; j0 < stride; j0 += ns) {
        const int base0 = (j0 / ns) * span;
        for (int k = 0; k < ns; ++k) {
          const int j = j0 + k;
          const cplx* tw = st.twiddle.data() + std::size_t(k) * r;
          a[0] = in[j];
          for (int t = 1; t < r; ++t) a[t] = in[j + t * stride] * tw[t];
          small_dft(a, b, st);
          const int base = base0 + k;
          for (int t = 0; t < r; ++t) out[base + t * ns] = b[t];
        }
      }
      std::swap(in, out);
    }
    if (in != x) std::copy_n(in, n_, x);
  }

 private:
  struct Stage {
    int radix;
    int ns;
    std::vector<cplx> twiddle;  // (k, t)
    std::vector<cplx> roots;    // w_r^q
  };

  // exp(s 2 pi i k / n): exact on the axes, elsewhere cos and sin of 2 pi k / n.
  cplx root(long k, long n) const {
    k %= n;
    if (k == 0) return {1.0, 0.0};
    if (4 * k == n) return {0.0, sign_};
    if (2 * k == n) return {-1.0, 0.0};
    if (4 * k == 3 * n) return {0.0, -sign_};
    const double angle = 2.0 * std::numbers::pi * static_cast<double>(k) / static_cast<double>(n);
    return {std::cos(angle), sign_ * std::sin(angle)};
  }

  // out[q] = sum_t in[t] w_r^(t q).
  void small_dft(const cplx* in, cplx* out, const Stage& st) const {
    const int r = st.radix;
    if (r == 2) {
      out[0] = in[0] + in[1];
      out[1] = in[0] - in[1];
      return;
    }
    if (r == 4) {
      const cplx s02 = in[0] + in[2], d02 = in[0] - in[2];
      const cplx s13 = in[1] + in[3], d13 = in[1] - in[3];
      const cplx j_d13(-sign_ * d13.imag(), sign_ * d13.real());  // s i (in1 - in3)
      out[0] = s02 + s13;
      out[1] = d02 + j_d13;
      out[2] = s02 - s13;
      out[3] = d02 - j_d13;
      return;
    }
    if (r == 3) {
      const cplx w = st.roots[1];
      const cplx s12 = in[1] + in[2];
      const cplx d12 = in[1] - in[2];
      const cplx m = in[0] + w.real() * s12;
      const cplx rot(-w.imag() * d12.imag(), w.imag() * d12.real());  // i Im(w) (in1 - in2)
      out[0] = in[0] + s12;
      out[1] = m + rot;
      out[2] = m - rot;
      return;
    }
    if (r > 63) {
      for (int q = 0; q < r; ++q) {
        cplx v = in[0];
        for (int t = 1; t < r; ++t) v += in[t] * st.roots[(static_cast<long>(t) * q) % r];
        out[q] = v;
      }
      return;
    }
    // Odd r: pairs t, r - t share cos and have opposite sin, so sum and difference halve the work.
    const int half = r / 2;
    cplx sum[32], dif[32];
    for (int t = 1; t <= half; ++t) {
      sum[t] = in[t] + in[r - t];
      dif[t] = in[t] - in[r - t];
    }
    cplx dc = in[0];
    for (int t = 1; t <= half; ++t) dc += sum[t];
    out[0] = dc;
    for (int q = 1; q <= half; ++q) {
      cplx re = in[0];
      double im_re = 0.0, im_im = 0.0;
      int tq = 0;
      for (int t = 1; t <= half; ++t) {
        tq += q;
        if (tq >= r) tq -= r;
        const cplx w = st.roots[tq];
        re += w.real() * sum[t];
        im_re += w.imag() * dif[t].real();
        im_im += w.imag() * dif[t].imag();
      }
      const cplx rot(-im_im, im_re);  // i * sum Im(w) dif
      out[q] = re + rot;
      out[r - q] = re - rot;
    }
  }

  int n_;
  double sign_;
  int r_max_ = 1;
  std::vector<Stage> stages_;
};

// Per-thread scratch for one line and its work array.
cplx* scratch(std::size_t n) {
  thread_local std::vector<cplx> buffer;
  if (buffer.size() < 2 * n) buffer.resize(2 * n);
  return buffer.data();
}

struct Dimension {
  int length;
  int stride;
};

// In-place batched complex transforms of rank 1 or 2 (dims outer first).
class ComplexPlan final : public ComplexFftPlan {
 public:
  ComplexPlan(std::vector<Dimension> dims, Dimension batch, FftSign sign, double scale)
      : dims_(std::move(dims)), batch_(batch), scale_(scale), size_(1 + std::size_t(batch.length - 1) * batch.stride) {
    for (const Dimension& d : dims_) {
      size_ += std::size_t(d.length - 1) * d.stride;
      lines_.emplace_back(d.length, sign);
    }
  }

  void execute(std::span<cplx> data) const override {
    if (data.size() < size_) throw std::invalid_argument("FftwFft: array too small for the FFT layout");
    for (int b = 0; b < batch_.length; ++b) {
      cplx* base = data.data() + std::size_t(b) * batch_.stride;
      if (dims_.size() == 1) {
        transform_line(base, lines_[0], dims_[0].stride);
      } else {
        const Dimension& outer = dims_[0];
        const Dimension& inner = dims_[1];
        for (int o = 0; o < outer.length; ++o) transform_line(base + std::size_t(o) * outer.stride, lines_[1], inner.stride);
        for (int i = 0; i < inner.length; ++i) transform_line(base + std::size_t(i) * inner.stride, lines_[0], outer.stride);
      }
    }
    if (scale_ != 1.0) apply_scale(data);
  }

 private:
  static void transform_line(cplx* p, const Line& line, int stride) {
    const int n = line.size();
    cplx* buf = scratch(n);
    for (int i = 0; i < n; ++i) buf[i] = p[std::size_t(i) * stride];
    line.run(buf, buf + n);
    for (int i = 0; i < n; ++i) p[std::size_t(i) * stride] = buf[i];
  }

  void apply_scale(std::span<cplx> data) const {
    const Dimension outer = dims_.size() == 2 ? dims_[0] : Dimension{1, 0};
    const Dimension inner = dims_.back();
    for (int b = 0; b < batch_.length; ++b)
      for (int o = 0; o < outer.length; ++o)
        for (int i = 0; i < inner.length; ++i) {
          cplx& v = data[std::size_t(b) * batch_.stride + std::size_t(o) * outer.stride + std::size_t(i) * inner.stride];
          v = scale_ * v;
        }
  }

  std::vector<Dimension> dims_;
  Dimension batch_;
  double scale_;
  std::size_t size_;
  std::vector<Line> lines_;
};

int distance_of(const FftLayout& layout, int logical_length) {
  return layout.distance > 0 ? layout.distance : logical_length;
}

std::size_t extent(const FftLayout& layout, int logical_length) {
  return std::size_t(layout.howmany - 1) * distance_of(layout, logical_length) +
         std::size_t(logical_length - 1) * layout.stride + 1;
}

// Real input: y_k = scale * sum_n x_n exp(s 2 pi i k n / N), k = 0 .. N/2.
class RealToComplexPlan final : public RealToComplexFftPlan {
 public:
  RealToComplexPlan(const FftLayout& in, const FftLayout& out, FftSign sign, double scale)
      : in_(in), out_(out), scale_(scale), line_(in.length, sign) {}

  void execute(std::span<const double> in, std::span<cplx> out) const override {
    const int n = in_.length;
    if (in.size() < extent(in_, n) || out.size() < extent(out_, n / 2 + 1))
      throw std::invalid_argument("FftwFft: array too small for the FFT layout");
    cplx* buf = scratch(n);
    for (int b = 0; b < in_.howmany; ++b) {
      for (int i = 0; i < n; ++i) buf[i] = in[std::size_t(b) * distance_of(in_, n) + std::size_t(i) * in_.stride];
      line_.run(buf, buf + n);
      for (int k = 0; k <= n / 2; ++k) {
        const cplx v = buf[k];
        out[std::size_t(b) * distance_of(out_, n / 2 + 1) + std::size_t(k) * out_.stride] = scale_ != 1.0 ? scale_ * v : v;
      }
    }
  }

 private:
  FftLayout in_;
  FftLayout out_;
  double scale_;
  Line line_;
};

// Half spectrum in, real output: the Hermitian extension transformed, its real part scaled.
class ComplexToRealPlan final : public ComplexToRealFftPlan {
 public:
  ComplexToRealPlan(const FftLayout& in, const FftLayout& out, FftSign sign, double scale)
      : in_(in), out_(out), scale_(scale), line_(out.length, sign) {}

  void execute(std::span<const cplx> in, std::span<double> out) const override {
    const int n = out_.length;
    if (in.size() < extent(in_, n / 2 + 1) || out.size() < extent(out_, n))
      throw std::invalid_argument("FftwFft: array too small for the FFT layout");
    cplx* buf = scratch(n);
    for (int b = 0; b < out_.howmany; ++b) {
      const cplx* src = in.data() + std::size_t(b) * distance_of(in_, n / 2 + 1);
      for (int k = 0; k <= n / 2; ++k) buf[k] = src[std::size_t(k) * in_.stride];
      buf[0] = cplx(buf[0].real(), 0.0);
      if (n % 2 == 0) buf[n / 2] = cplx(buf[n / 2].real(), 0.0);
      for (int k = n / 2 + 1; k < n; ++k) buf[k] = std::conj(buf[n - k]);
      line_.run(buf, buf + n);
      for (int i = 0; i < n; ++i) {
        const double v = buf[i].real();
        out[std::size_t(b) * distance_of(out_, n) + std::size_t(i) * out_.stride] = scale_ != 1.0 ? scale_ * v : v;
      }
    }
  }

 private:
  FftLayout in_;
  FftLayout out_;
  double scale_;
  Line line_;
};

void check_layout(const FftLayout& layout) {
  if (layout.length < 1 || layout.howmany < 1 || layout.stride < 1 || layout.distance < 0)
    throw std::invalid_argument("FftwFft: invalid FFT layout");
}

}  // namespace

std::unique_ptr<ComplexFftPlan> FftwFft::plan_complex(const FftLayout& layout, FftSign sign, double scale) const {
  check_layout(layout);
  return std::make_unique<ComplexPlan>(std::vector<Dimension>{{layout.length, layout.stride}},
                                       Dimension{layout.howmany, distance_of(layout, layout.length)}, sign, scale);
}

std::unique_ptr<ComplexFftPlan> FftwFft::plan_complex_2d(const FftLayout2D& layout, FftSign sign, double scale) const {
  if (layout.outer_length < 1 || layout.inner_length < 1 || layout.howmany < 1 || layout.outer_stride < 1 ||
      layout.inner_stride < 1 || layout.distance < 1)
    throw std::invalid_argument("FftwFft: invalid 2D FFT layout");
  return std::make_unique<ComplexPlan>(
      std::vector<Dimension>{{layout.outer_length, layout.outer_stride}, {layout.inner_length, layout.inner_stride}},
      Dimension{layout.howmany, layout.distance}, sign, scale);
}

std::unique_ptr<RealToComplexFftPlan> FftwFft::plan_real_to_complex(const FftLayout& in, const FftLayout& out,
                                                                    FftSign sign, double scale) const {
  check_layout(in);
  if (out.howmany != in.howmany) throw std::invalid_argument("FftwFft: howmany mismatch");
  return std::make_unique<RealToComplexPlan>(in, FftLayout{in.length, out.howmany, out.stride, out.distance}, sign,
                                             scale);
}

std::unique_ptr<ComplexToRealFftPlan> FftwFft::plan_complex_to_real(const FftLayout& in, const FftLayout& out,
                                                                    FftSign sign, double scale) const {
  check_layout(out);
  if (out.howmany != in.howmany) throw std::invalid_argument("FftwFft: howmany mismatch");
  return std::make_unique<ComplexToRealPlan>(FftLayout{out.length, in.howmany, in.stride, in.distance}, out, sign,
                                             scale);
}

}  // namespace spodvr
