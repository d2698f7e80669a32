// Stand-in for the pocketfft header (mreineck/pocketfft, C++ header-only branch, pinned by the
// reference build at commit 4d865cba24359b05b37da4e75aee24498c3b78e7). That dependency is not
// shipped with the reference sources and cannot be fetched here, so this file provides the five
// entry points the reference calls -- c2c, r2c (one or several axes), c2r (one axis) and dct
// type 2 -- with pocketfft's signatures and semantics: strides in bytes, `forward` selects the
// sign of the exponent (e^{-2 pi i jk/n} forward), results multiplied by `fct`, no implicit
// normalisation, c2r ignores the imaginary parts that a real signal cannot have.
//
// The transforms are written from the mathematics: a Stockham autosort decimation-in-time FFT
// with radix 4, 2, 3, 5 passes and a direct DFT for any other prime factor, twiddles computed in
// double and rounded once, arithmetic in the data type like pocketfft. Results agree with
// numpy.fft (itself pocketfft) to float rounding, which the oracle tests check.
//
// This header is test infrastructure: it is compiled only into oracle/_ref, the CPU reference
// built from the reference sources, never into the product library.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace pocketfft {
namespace detail {

using shape_t = std::vector<std::size_t>;
using stride_t = std::vector<std::ptrdiff_t>;

template <class T>
class Plan1d {
 public:
  explicit Plan1d(std::size_t n) : n_(n) {
    if (n == 0) throw std::invalid_argument("pocketfft shim: zero length");
    std::size_t m = n;
    while (m % 4 == 0) { radix_.push_back(4); m /= 4; }
    while (m % 2 == 0) { radix_.push_back(2); m /= 2; }
    for (std::size_t p = 3; p * p <= m; p += 2) {
      while (m % p == 0) { radix_.push_back(p); m /= p; }
    }
    if (m > 1) radix_.push_back(m);
    tw_.resize(n);
    const double two_pi = 6.283185307179586476925286766559;
    for (std::size_t k = 0; k < n; ++k) {
      const double a = two_pi * double(k) / double(n);
      tw_[k] = std::complex<T>(T(std::cos(a)), T(-std::sin(a)));  // e^{-2 pi i k / n}
    }
  }

  // In-place transform of one contiguous line; scratch holds n values.
  void exec(std::complex<T>* data, std::complex<T>* scratch, bool forward) const {
    std::complex<T>* src = data;
    std::complex<T>* dst = scratch;
    std::size_t ns = 1;
    for (std::size_t r : radix_) {
      pass(src, dst, ns, r, forward);
      std::swap(src, dst);
      ns *= r;
    }
    if (src != data) std::memcpy(data, src, n_ * sizeof(std::complex<T>));
  }

  std::size_t size() const { return n_; }

 private:
  std::complex<T> w(std::size_t k, bool forward) const {
    const std::complex<T> v = tw_[k % n_];
    return forward ? v : std::conj(v);
  }

  void pass(const std::complex<T>* in, std::complex<T>* out, std::size_t ns, std::size_t r,
            bool forward) const {
    const std::size_t n = n_;
    const std::size_t m = n / r;          // butterflies in this pass
    const std::size_t step = n / (ns * r);  // twiddle index step for k * q
    std::complex<T> v[64];
    std::vector<std::complex<T>> big;
    std::complex<T>* vp = v;
    if (r > 64) {
      big.resize(r);
      vp = big.data();
    }
    for (std::size_t j = 0; j < m; ++j) {
      const std::size_t k = j % ns;
      for (std::size_t q = 0; q < r; ++q) {
        std::complex<T> x = in[j + q * m];
        if (q && k) x *= w(k * q * step, forward);
        vp[q] = x;
      }
      butterfly(vp, r, forward);
      const std::size_t base = (j / ns) * ns * r + k;
      for (std::size_t q = 0; q < r; ++q) out[base + q * ns] = vp[q];
    }
  }

  void butterfly(std::complex<T>* v, std::size_t r, bool forward) const {
    const T s = forward ? T(-1) : T(1);  // sign of the exponent
    if (r == 2) {
      const std::complex<T> a = v[0], b = v[1];
      v[0] = a + b;
      v[1] = a - b;
    } else if (r == 4) {
      const std::complex<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
      const std::complex<T> b0 = v[1] + v[3], b1 = v[1] - v[3];
      const std::complex<T> jb1(-s * b1.imag(), s * b1.real());  // i*s*b1
      v[0] = a0 + b0;
      v[2] = a0 - b0;
      v[1] = a1 + jb1;
      v[3] = a1 - jb1;
    } else if (r == 3) {
      const T c = T(-0.5);
      const T sn = s * T(0.86602540378443864676);
      const std::complex<T> t1 = v[1] + v[2];
      const std::complex<T> t2 = v[0] + c * t1;
      const std::complex<T> t3 = v[1] - v[2];
      const std::complex<T> t4(-sn * t3.imag(), sn * t3.real());
      v[0] = v[0] + t1;
      v[1] = t2 + t4;
      v[2] = t2 - t4;
    } else {
      // Direct DFT of a prime length, twiddles from the plan's table.
      std::complex<T> out[64];
      std::vector<std::complex<T>> big;
      std::complex<T>* o = out;
      if (r > 64) {
        big.resize(r);
        o = big.data();
      }
      const std::size_t stride = n_ / r;
      for (std::size_t q = 0; q < r; ++q) {
        std::complex<T> acc = v[0];
        for (std::size_t p = 1; p < r; ++p) acc += v[p] * w(((p * q) % r) * stride, forward);
        o[q] = acc;
      }
      for (std::size_t q = 0; q < r; ++q) v[q] = o[q];
    }
  }

  std::size_t n_;
  std::vector<std::size_t> radix_;
  std::vector<std::complex<T>> tw_;
};

// Offsets (in elements of `elem` bytes) of the first element of every line along `axis`.
inline std::vector<std::ptrdiff_t> line_bases(const shape_t& shape, const stride_t& stride,
                                              std::size_t axis, std::size_t elem) {
  std::vector<std::ptrdiff_t> bases{0};
  for (std::size_t d = 0; d < shape.size(); ++d) {
    if (d == axis) continue;
    std::vector<std::ptrdiff_t> next;
    next.reserve(bases.size() * shape[d]);
    for (std::ptrdiff_t b : bases) {
      for (std::size_t i = 0; i < shape[d]; ++i)
        next.push_back(b + std::ptrdiff_t(i) * stride[d] / std::ptrdiff_t(elem));
    }
    bases.swap(next);
  }
  return bases;
}

constexpr std::size_t kBlock = 16;  // lines gathered together for cache-friendly strided access

// Complex transform along one axis, out of place allowed (in may equal out).
template <class T>
void c2c_axis(const shape_t& shape, const stride_t& sin, const stride_t& sout, std::size_t axis,
              bool forward, const std::complex<T>* in, std::complex<T>* out, T fct,
              std::size_t nthreads) {
  const std::size_t n = shape[axis];
  const Plan1d<T> plan(n);
  const auto bin = line_bases(shape, sin, axis, sizeof(std::complex<T>));
  const auto bout = line_bases(shape, sout, axis, sizeof(std::complex<T>));
  const std::ptrdiff_t si = sin[axis] / std::ptrdiff_t(sizeof(std::complex<T>));
  const std::ptrdiff_t so = sout[axis] / std::ptrdiff_t(sizeof(std::complex<T>));
  const std::ptrdiff_t blocks = std::ptrdiff_t((bin.size() + kBlock - 1) / kBlock);
#pragma omp parallel num_threads(int(std::max<std::size_t>(nthreads, 1)))
  {
    std::vector<std::complex<T>> buf(kBlock * n);
    std::vector<std::complex<T>> scratch(n);
#pragma omp for schedule(static)
    for (std::ptrdiff_t blk = 0; blk < blocks; ++blk) {
      const std::size_t l0 = std::size_t(blk) * kBlock;
      const std::size_t nl = std::min(kBlock, bin.size() - l0);
      for (std::size_t p = 0; p < n; ++p)
        for (std::size_t l = 0; l < nl; ++l) buf[l * n + p] = in[bin[l0 + l] + std::ptrdiff_t(p) * si];
      for (std::size_t l = 0; l < nl; ++l) {
        plan.exec(buf.data() + l * n, scratch.data(), forward);
        if (fct != T(1))
          for (std::size_t p = 0; p < n; ++p) buf[l * n + p] *= fct;
      }
      for (std::size_t p = 0; p < n; ++p)
        for (std::size_t l = 0; l < nl; ++l) out[bout[l0 + l] + std::ptrdiff_t(p) * so] = buf[l * n + p];
    }
  }
}

template <class T>
void c2c(const shape_t& shape, const stride_t& stride_in, const stride_t& stride_out,
         const shape_t& axes, bool forward, const std::complex<T>* data_in,
         std::complex<T>* data_out, T fct, std::size_t nthreads = 1) {
  if (axes.empty()) return;
  for (std::size_t i = 0; i < axes.size(); ++i) {
    const bool first = i == 0;
    c2c_axis<T>(shape, first ? stride_in : stride_out, stride_out, axes[i], forward,
                first ? data_in : data_out, data_out, first ? fct : T(1), nthreads);
  }
}

// Real input along `axis` -> half spectrum (n/2 + 1 bins) along that axis.
template <class T>
void r2c(const shape_t& shape_in, const stride_t& stride_in, const stride_t& stride_out,
         std::size_t axis, bool forward, const T* data_in, std::complex<T>* data_out, T fct,
         std::size_t nthreads = 1) {
  const std::size_t n = shape_in[axis];
  const std::size_t h = n / 2 + 1;
  shape_t shape_out = shape_in;
  shape_out[axis] = h;
  const Plan1d<T> plan(n);
  const auto bin = line_bases(shape_in, stride_in, axis, sizeof(T));
  const auto bout = line_bases(shape_out, stride_out, axis, sizeof(std::complex<T>));
  const std::ptrdiff_t si = stride_in[axis] / std::ptrdiff_t(sizeof(T));
  const std::ptrdiff_t so = stride_out[axis] / std::ptrdiff_t(sizeof(std::complex<T>));
  const std::ptrdiff_t blocks = std::ptrdiff_t((bin.size() + kBlock - 1) / kBlock);
#pragma omp parallel num_threads(int(std::max<std::size_t>(nthreads, 1)))
  {
    std::vector<std::complex<T>> buf(kBlock * n);
    std::vector<std::complex<T>> scratch(n);
#pragma omp for schedule(static)
    for (std::ptrdiff_t blk = 0; blk < blocks; ++blk) {
      const std::size_t l0 = std::size_t(blk) * kBlock;
      const std::size_t nl = std::min(kBlock, bin.size() - l0);
      for (std::size_t p = 0; p < n; ++p)
        for (std::size_t l = 0; l < nl; ++l)
          buf[l * n + p] = std::complex<T>(data_in[bin[l0 + l] + std::ptrdiff_t(p) * si], T(0));
      for (std::size_t l = 0; l < nl; ++l) {
        plan.exec(buf.data() + l * n, scratch.data(), forward);
        for (std::size_t p = 0; p < h; ++p) buf[l * n + p] *= fct;
      }
      for (std::size_t p = 0; p < h; ++p)
        for (std::size_t l = 0; l < nl; ++l)
          data_out[bout[l0 + l] + std::ptrdiff_t(p) * so] = buf[l * n + p];
    }
  }
}

template <class T>
void r2c(const shape_t& shape_in, const stride_t& stride_in, const stride_t& stride_out,
         const shape_t& axes, bool forward, const T* data_in, std::complex<T>* data_out, T fct,
         std::size_t nthreads = 1) {
  if (axes.empty()) return;
  r2c<T>(shape_in, stride_in, stride_out, axes.back(), forward, data_in, data_out, fct, nthreads);
  if (axes.size() > 1) {
    shape_t shape_out = shape_in;
    shape_out[axes.back()] = shape_in[axes.back()] / 2 + 1;
    const shape_t rest(axes.begin(), axes.end() - 1);
    c2c<T>(shape_out, stride_out, stride_out, rest, forward, data_out, data_out, T(1), nthreads);
  }
}

// Half spectrum along `axis` -> real output of length shape_out[axis].
template <class T>
void c2r(const shape_t& shape_out, const stride_t& stride_in, const stride_t& stride_out,
         std::size_t axis, bool forward, const std::complex<T>* data_in, T* data_out, T fct,
         std::size_t nthreads = 1) {
  const std::size_t n = shape_out[axis];
  const std::size_t h = n / 2 + 1;
  shape_t shape_in = shape_out;
  shape_in[axis] = h;
  const Plan1d<T> plan(n);
  const auto bin = line_bases(shape_in, stride_in, axis, sizeof(std::complex<T>));
  const auto bout = line_bases(shape_out, stride_out, axis, sizeof(T));
  const std::ptrdiff_t si = stride_in[axis] / std::ptrdiff_t(sizeof(std::complex<T>));
  const std::ptrdiff_t so = stride_out[axis] / std::ptrdiff_t(sizeof(T));
  const std::ptrdiff_t blocks = std::ptrdiff_t((bin.size() + kBlock - 1) / kBlock);
#pragma omp parallel num_threads(int(std::max<std::size_t>(nthreads, 1)))
  {
    std::vector<std::complex<T>> buf(kBlock * n);
    std::vector<std::complex<T>> scratch(n);
#pragma omp for schedule(static)
    for (std::ptrdiff_t blk = 0; blk < blocks; ++blk) {
      const std::size_t l0 = std::size_t(blk) * kBlock;
      const std::size_t nl = std::min(kBlock, bin.size() - l0);
      for (std::size_t p = 0; p < h; ++p)
        for (std::size_t l = 0; l < nl; ++l) buf[l * n + p] = data_in[bin[l0 + l] + std::ptrdiff_t(p) * si];
      for (std::size_t l = 0; l < nl; ++l) {
        std::complex<T>* line = buf.data() + l * n;
        // Hermitian completion; the imaginary parts of bins 0 and n/2 drop out of the real part.
        for (std::size_t p = h; p < n; ++p) line[p] = std::conj(line[n - p]);
        plan.exec(line, scratch.data(), forward);
      }
      for (std::size_t p = 0; p < n; ++p)
        for (std::size_t l = 0; l < nl; ++l)
          data_out[bout[l0 + l] + std::ptrdiff_t(p) * so] = buf[l * n + p].real() * fct;
    }
  }
}

// DCT of type 2 along the given axes, FFTW's REDFT10 convention y_k = 2 sum x_j cos(pi k (2j+1)
// / 2n), times fct; `ortho` is not supported (the reference never sets it).
template <class T>
void dct(const shape_t& shape, const stride_t& stride_in, const stride_t& stride_out,
         const shape_t& axes, int type, const T* data_in, T* data_out, T fct, bool ortho,
         std::size_t nthreads = 1) {
  if (type != 2 || ortho) throw std::invalid_argument("pocketfft shim: only unnormalised DCT-II");
  (void)nthreads;
  for (std::size_t i = 0; i < axes.size(); ++i) {
    const std::size_t axis = axes[i];
    const std::size_t n = shape[axis];
    const stride_t& sin = i == 0 ? stride_in : stride_out;
    const T* in = i == 0 ? data_in : data_out;
    const auto bin = line_bases(shape, sin, axis, sizeof(T));
    const auto bout = line_bases(shape, stride_out, axis, sizeof(T));
    const std::ptrdiff_t si = sin[axis] / std::ptrdiff_t(sizeof(T));
    const std::ptrdiff_t so = stride_out[axis] / std::ptrdiff_t(sizeof(T));
    std::vector<double> line(n);
    const double pi = 3.141592653589793238462643383279;
    for (std::size_t l = 0; l < bin.size(); ++l) {
      for (std::size_t j = 0; j < n; ++j) line[j] = double(in[bin[l] + std::ptrdiff_t(j) * si]);
      for (std::size_t k = 0; k < n; ++k) {
        double acc = 0;
        for (std::size_t j = 0; j < n; ++j) acc += line[j] * std::cos(pi * double(k) * (2.0 * j + 1.0) / (2.0 * n));
        data_out[bout[l] + std::ptrdiff_t(k) * so] = T(2.0 * acc) * (i == 0 ? fct : T(1));
      }
    }
  }
}

}  // namespace detail

using detail::c2c;
using detail::c2r;
using detail::dct;
using detail::r2c;
using detail::shape_t;
using detail::stride_t;

}  // namespace pocketfft
