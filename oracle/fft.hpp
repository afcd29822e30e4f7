// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle; never linked into the product.
//
// Mixed-radix (2,3,4,5) Stockham FFT used by the oracle in place of FFTW 3.3.8, the
// un-vendored third-party library the reference calls (cubefft.f90:21-37,
// pencil_fft.f90:327-338).  Convention follows FFTW: forward e^{-i}, backward e^{+i},
// both unnormalised; r2c keeps n/2+1 outputs along the fastest (x) axis.
// The FFT is cross-checked against numpy.fft (pocketfft) by the oracle tests.
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace oracle {

inline std::vector<int> fft_factor(int n) {
  std::vector<int> r;
  while (n % 4 == 0) { r.push_back(4); n /= 4; }
  while (n % 2 == 0) { r.push_back(2); n /= 2; }
  while (n % 3 == 0) { r.push_back(3); n /= 3; }
  while (n % 5 == 0) { r.push_back(5); n /= 5; }
  if (n != 1) throw std::runtime_error("fft size is not 2,3,5-smooth");
  return r;
}

// One 1D plan: radices plus per-stage twiddles e^{sign 2 pi i r (j mod Ns)/(Ns R)}.
template <class T>
struct Plan1D {
  int n = 0;
  int sign = -1;
  std::vector<int> rad;
  std::vector<std::complex<T>> tw;  // concatenated per stage: for j in [0,Ns), r in [1,R)
  std::vector<size_t> twoff;
  void init(int n_, int sign_) {
    n = n_;
    sign = sign_;
    rad = fft_factor(n);
    tw.clear();
    twoff.clear();
    int Ns = 1;
    for (int R : rad) {
      twoff.push_back(tw.size());
      for (int j = 0; j < Ns; ++j)
        for (int r = 1; r < R; ++r) {
          double ang = sign * 2.0 * M_PI * (double)r * (double)j / (double)(Ns * R);
          tw.push_back(std::complex<T>((T)std::cos(ang), (T)std::sin(ang)));
        }
      Ns *= R;
    }
  }
  // In-place transform of `a` (length n) using `scratch` (length n).
  void exec(std::complex<T>* a, std::complex<T>* scratch) const {
    std::complex<T>* in = a;
    std::complex<T>* out = scratch;
    int Ns = 1;
    const T s3 = (T)(sign * std::sqrt(3.0) / 2.0);
    const double c5a = std::cos(2 * M_PI / 5), c5b = std::cos(4 * M_PI / 5);
    const double s5a = std::sin(2 * M_PI / 5), s5b = std::sin(4 * M_PI / 5);
    for (size_t st = 0; st < rad.size(); ++st) {
      const int R = rad[st];
      const int m = n / R;
      const std::complex<T>* w = tw.data() + twoff[st];
      for (int j = 0; j < m; ++j) {
        std::complex<T> v[5];
        const int jm = j % Ns;
        for (int r = 0; r < R; ++r) v[r] = in[j + r * m];
        for (int r = 1; r < R; ++r) v[r] *= w[jm * (R - 1) + (r - 1)];
        std::complex<T> y[5];
        if (R == 2) {
          y[0] = v[0] + v[1];
          y[1] = v[0] - v[1];
        } else if (R == 4) {
          std::complex<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
          std::complex<T> b0 = v[1] + v[3], b1 = v[1] - v[3];
          // multiply b1 by sign*i
          std::complex<T> jb1 = (sign < 0) ? std::complex<T>(b1.imag(), -b1.real())
                                           : std::complex<T>(-b1.imag(), b1.real());
          y[0] = a0 + b0;
          y[2] = a0 - b0;
          y[1] = a1 + jb1;
          y[3] = a1 - jb1;
        } else if (R == 3) {
          std::complex<T> t = v[1] + v[2];
          std::complex<T> d = v[1] - v[2];
          std::complex<T> m0 = v[0] - (T)0.5 * t;
          std::complex<T> id(-d.imag() * s3, d.real() * s3);  // i*s3*d
          y[0] = v[0] + t;
          y[1] = m0 + id;
          y[2] = m0 - id;
        } else {  // R == 5, direct small DFT
          for (int k = 0; k < 5; ++k) {
            std::complex<double> acc(0, 0);
            for (int r = 0; r < 5; ++r) {
              double ang = sign * 2.0 * M_PI * (double)((r * k) % 5) / 5.0;
              acc += std::complex<double>(v[r].real(), v[r].imag()) *
                     std::complex<double>(std::cos(ang), std::sin(ang));
            }
            y[k] = std::complex<T>((T)acc.real(), (T)acc.imag());
          }
          (void)c5a; (void)c5b; (void)s5a; (void)s5b;
        }
        const int idxD = (j / Ns) * Ns * R + jm;
        for (int r = 0; r < R; ++r) out[idxD + r * Ns] = y[r];
      }
      std::swap(in, out);
      Ns *= R;
    }
    if (in != a)
      for (int i = 0; i < n; ++i) a[i] = in[i];
  }
};

// 3D real-to-complex forward transform of r[n][n][n] (z,y,x; x fastest) into
// c[n][n][n/2+1], unnormalised.
template <class T>
void rfft3(int n, const T* r, std::complex<T>* c) {
  const int nh = n / 2 + 1;
  Plan1D<T> p;
  p.init(n, -1);
  std::vector<std::complex<T>> buf(n), scr(n);
  for (int64_t zy = 0; zy < (int64_t)n * n; ++zy) {
    for (int x = 0; x < n; ++x) buf[x] = std::complex<T>(r[zy * n + x], 0);
    p.exec(buf.data(), scr.data());
    for (int x = 0; x < nh; ++x) c[zy * nh + x] = buf[x];
  }
  for (int z = 0; z < n; ++z)
    for (int x = 0; x < nh; ++x) {
      for (int y = 0; y < n; ++y) buf[y] = c[((int64_t)z * n + y) * nh + x];
      p.exec(buf.data(), scr.data());
      for (int y = 0; y < n; ++y) c[((int64_t)z * n + y) * nh + x] = buf[y];
    }
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nh; ++x) {
      for (int z = 0; z < n; ++z) buf[z] = c[((int64_t)z * n + y) * nh + x];
      p.exec(buf.data(), scr.data());
      for (int z = 0; z < n; ++z) c[((int64_t)z * n + y) * nh + x] = buf[z];
    }
}

// 3D complex-to-real backward transform, unnormalised (FFTW c2r convention: the
// half spectrum is read as a Hermitian-symmetric full spectrum).  c is destroyed.
template <class T>
void irfft3(int n, std::complex<T>* c, T* r) {
  const int nh = n / 2 + 1;
  Plan1D<T> p;
  p.init(n, +1);
  std::vector<std::complex<T>> buf(n), scr(n);
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nh; ++x) {
      for (int z = 0; z < n; ++z) buf[z] = c[((int64_t)z * n + y) * nh + x];
      p.exec(buf.data(), scr.data());
      for (int z = 0; z < n; ++z) c[((int64_t)z * n + y) * nh + x] = buf[z];
    }
  for (int z = 0; z < n; ++z)
    for (int x = 0; x < nh; ++x) {
      for (int y = 0; y < n; ++y) buf[y] = c[((int64_t)z * n + y) * nh + x];
      p.exec(buf.data(), scr.data());
      for (int y = 0; y < n; ++y) c[((int64_t)z * n + y) * nh + x] = buf[y];
    }
  for (int64_t zy = 0; zy < (int64_t)n * n; ++zy) {
    for (int x = 0; x < nh; ++x) buf[x] = c[zy * nh + x];
    buf[0] = std::complex<T>(buf[0].real(), 0);
    if (n % 2 == 0) buf[n / 2] = std::complex<T>(buf[n / 2].real(), 0);
    for (int x = nh; x < n; ++x) buf[x] = std::conj(buf[n - x]);
    p.exec(buf.data(), scr.data());
    for (int x = 0; x < n; ++x) r[zy * n + x] = buf[x].real();
  }
}

}  // namespace oracle
