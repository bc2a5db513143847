// Host-side plans for the line FFTs of line_fft.cuh: the plan construction
// of the pocketfft C++ library (NumPy 2.x's FFT), restated so that the
// device transforms use the same factors, the same twiddle values and the
// same Bluestein chirp as numpy.fft, bit for bit:
//
// * pocketfft_c: Cooley-Tukey when n < 50 or its largest prime factor p has
//   p² ≤ n, otherwise Bluestein when 1.5 · 2 · cost(n2) < cost(n) with
//   n2 = the smallest 11-smooth length ≥ 2n − 1;
// * cfftp::factorize: 8s, then 4s, a remaining 2 swapped to the front, then
//   odd primes in increasing order;
// * cfftp::comp_twiddle: per pass, w[(j−1)(ido−1) + i−1] = e^{2πi·j·l1·i/n},
//   plus the p roots of a generic pass (p > 11);
// * sincos_2pibyn: e^{2πik/n} as the product of two table entries
//   v1[k & mask] · v2[k >> shift], the tables filled from cos/sin of octant-
//   reduced angles (the angle step π/(4n) computed in long double);
// * fftblue: chirp b_k = e^{iπk²/n} read from the 2n-table, and its zero-
//   padded copy scaled by 1/n2 (its transform is computed on the device).
//
// Only the arithmetic that the library does on the host side of a plan is
// here; the transforms themselves run on the device.
#pragma once

#include <cmath>
#include <cstddef>
#include <utility>
#include <vector>

namespace ertm {
namespace fftplan {

struct CxH {
  double r, i;
};

class SinCos2PiByN {
 public:
  explicit SinCos2PiByN(size_t n) : n_(n) {
    constexpr long double pi = 3.141592653589793238462643383279502884197L;
    const double ang = double(0.25L * pi / (long double)n);
    const size_t nval = (n + 2) / 2;
    shift_ = 1;
    while ((size_t(1) << shift_) * (size_t(1) << shift_) < nval) ++shift_;
    mask_ = (size_t(1) << shift_) - 1;
    v1_.resize(mask_ + 1);
    v1_[0] = {1.0, 0.0};
    for (size_t i = 1; i < v1_.size(); ++i) v1_[i] = calc(i, n, ang);
    v2_.resize((nval + mask_) / (mask_ + 1));
    v2_[0] = {1.0, 0.0};
    for (size_t i = 1; i < v2_.size(); ++i) v2_[i] = calc(i * (mask_ + 1), n, ang);
  }

  CxH operator[](size_t idx) const {
    if (2 * idx <= n_) {
      const CxH x1 = v1_[idx & mask_], x2 = v2_[idx >> shift_];
      return {x1.r * x2.r - x1.i * x2.i, x1.r * x2.i + x1.i * x2.r};
    }
    idx = n_ - idx;
    const CxH x1 = v1_[idx & mask_], x2 = v2_[idx >> shift_];
    return {x1.r * x2.r - x1.i * x2.i, -(x1.r * x2.i + x1.i * x2.r)};
  }

 private:
  // e^{2πix/n} for x in [0, n): the angle x·π/(4n)·8 reduced to the first
  // octant, cos/sin swapped and negated per octant
  static CxH calc(size_t x, size_t n, double ang) {
    x <<= 3;
    if (x < 4 * n) {
      if (x < 2 * n) {
        if (x < n) return {std::cos(double(x) * ang), std::sin(double(x) * ang)};
        return {std::sin(double(2 * n - x) * ang), std::cos(double(2 * n - x) * ang)};
      }
      x -= 2 * n;
      if (x < n) return {-std::sin(double(x) * ang), std::cos(double(x) * ang)};
      return {-std::cos(double(2 * n - x) * ang), std::sin(double(2 * n - x) * ang)};
    }
    x = 8 * n - x;
    if (x < 2 * n) {
      if (x < n) return {std::cos(double(x) * ang), -std::sin(double(x) * ang)};
      return {std::sin(double(2 * n - x) * ang), -std::cos(double(2 * n - x) * ang)};
    }
    x -= 2 * n;
    if (x < n) return {-std::sin(double(x) * ang), -std::cos(double(x) * ang)};
    return {-std::cos(double(2 * n - x) * ang), -std::sin(double(2 * n - x) * ang)};
  }

  size_t n_, mask_ = 0, shift_ = 0;
  std::vector<CxH> v1_, v2_;
};

inline size_t largest_prime_factor(size_t n) {
  size_t res = 1;
  while ((n & 1) == 0) {
    res = 2;
    n >>= 1;
  }
  for (size_t x = 3; x * x <= n; x += 2)
    while (n % x == 0) {
      res = x;
      n /= x;
    }
  if (n > 1) res = n;
  return res;
}

inline double cost_guess(size_t n) {
  constexpr double lfp = 1.1;   // penalty of the generic pass
  const size_t ni = n;
  double result = 0.0;
  while ((n & 1) == 0) {
    result += 2;
    n >>= 1;
  }
  for (size_t x = 3; x * x <= n; x += 2)
    while (n % x == 0) {
      result += (x <= 5) ? double(x) : lfp * double(x);
      n /= x;
    }
  if (n > 1) result += (n <= 5) ? double(n) : lfp * double(n);
  return result * double(ni);
}

// smallest 2^a 3^b 5^c 7^d 11^e ≥ n
inline size_t good_size_cmplx(size_t n) {
  if (n <= 12) return n;
  size_t bestfac = 2 * n;
  for (size_t f11 = 1; f11 < bestfac; f11 *= 11)
    for (size_t f117 = f11; f117 < bestfac; f117 *= 7)
      for (size_t f1175 = f117; f1175 < bestfac; f1175 *= 5) {
        size_t x = f1175;
        while (x < n) x *= 2;
        for (;;) {
          if (x < n) {
            x *= 3;
          } else if (x > n) {
            if (x < bestfac) bestfac = x;
            if (x & 1) break;
            x >>= 1;
          } else {
            return n;
          }
        }
      }
  return bestfac;
}

// Factors and twiddles of a Cooley-Tukey length (cfftp).
struct CooleyTukey {
  size_t n = 0;
  std::vector<int> fct, twoff, twsoff;
  std::vector<CxH> tw;

  explicit CooleyTukey(size_t len) : n(len) {
    if (n <= 1) return;
    size_t l = n;
    while ((l & 7) == 0) {
      fct.push_back(8);
      l >>= 3;
    }
    while ((l & 3) == 0) {
      fct.push_back(4);
      l >>= 2;
    }
    if ((l & 1) == 0) {
      l >>= 1;
      fct.push_back(2);
      std::swap(fct.front(), fct.back());
    }
    for (size_t d = 3; d * d <= l; d += 2)
      while (l % d == 0) {
        fct.push_back((int)d);
        l /= d;
      }
    if (l > 1) fct.push_back((int)l);
    const SinCos2PiByN comp(n);
    size_t l1 = 1;
    for (int ip : fct) {
      const size_t ido = n / (l1 * ip);
      twoff.push_back((int)tw.size());
      for (int j = 1; j < ip; ++j)
        for (size_t i = 1; i < ido; ++i) tw.push_back(comp[j * l1 * i]);
      twsoff.push_back((int)tw.size());
      if (ip > 11)
        for (int j = 0; j < ip; ++j) tw.push_back(comp[j * l1 * ido]);
      l1 *= ip;
    }
  }
};

// The library's choice between Cooley-Tukey and Bluestein for length n.
inline bool use_bluestein(size_t n) {
  const size_t tmp = n < 50 ? 0 : largest_prime_factor(n);
  if (tmp * tmp <= n) return false;
  const double comp1 = cost_guess(n);
  double comp2 = 2 * cost_guess(good_size_cmplx(2 * n - 1));
  comp2 *= 1.5;   // the library's fudge factor
  return comp2 < comp1;
}

// Bluestein chirp b_k (k < n) and the zero-padded, 1/n2-scaled kernel whose
// forward transform (length n2) gives the convolution weights.
inline void bluestein_chirp(size_t n, size_t n2, std::vector<CxH>& bk, std::vector<CxH>& kernel) {
  const SinCos2PiByN tmp(2 * n);
  bk.assign(n, CxH{0.0, 0.0});
  bk[0] = {1.0, 0.0};
  size_t coeff = 0;
  for (size_t m = 1; m < n; ++m) {
    coeff += 2 * m - 1;
    if (coeff >= 2 * n) coeff -= 2 * n;
    bk[m] = tmp[coeff];
  }
  const double xn2 = 1.0 / double(n2);
  kernel.assign(n2, CxH{0.0, 0.0});
  kernel[0] = {bk[0].r * xn2, bk[0].i * xn2};
  for (size_t m = 1; m < n; ++m) kernel[m] = kernel[n2 - m] = {bk[m].r * xn2, bk[m].i * xn2};
}

}  // namespace fftplan
}  // namespace ertm
