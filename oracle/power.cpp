// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle; never linked into the product.
//
// Restatement of CUBE's power-spectrum measurement for one image (nn=1):
//   utilities/cicpower.f90:76-98    CIC density of the ZIPX particles on an nw^3 mesh
//                                   (nw = ng*nic, parameters.f90:73 with FFTFINE)
//   utilities/cicpower.f90:107-150  periodic fold of the one-cell halo
//   utilities/cicpower.f90:165-181  delta = rho / (sum(rho)/nw^3) - 1
//   utilities/powerspectrum.f90:140-210  auto_power: forward FFT / nw^3, |delta_k|^2 in
//                                   linear bins nint(|k|), shot noise with the window
//                                   C1k of n_interp, normalisation
//   utilities/powerspectrum.f90:212-259  pk_correction: alias integral with n_int
//                                   images, xi(5) = xi(4)/<W^2 P>/P
// Arithmetic kinds follow the reference: positions, weights, the binned sums and the
// alias integral in real(4); the mean in real(8).  Two stand-ins: the FFT is the
// oracle's own (fft.hpp, here in double, rounded to float as FFTW's single-precision
// output would be), and with `fixed` the density is summed as int64 fixed point
// (round(w*2^40)), the library's deterministic mode, instead of in particle order.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "../include/cube_gpu.h"
#include "fft.hpp"

namespace opower {

struct PGeo {
  int64_t nc, nt, nnt;
  int izipx;
  double x_res;
};

static PGeo pgeo(const cube_params* p) {
  PGeo g;
  g.nc = p->ng / p->ratio_cs;
  g.nnt = p->nnt;
  g.nt = g.nc / g.nnt;
  g.izipx = p->izipx;
  g.x_res = std::ldexp(1.0, -8 * g.izipx);
  return g;
}

static inline int64_t wrap(int64_t a, int64_t n) {
  a %= n;
  return a < 0 ? a + n : a;
}

// gcc's integer power (libgcc __powisf2), which gfortran uses for real**integer.
static inline float powi(float x, int m) {
  unsigned n = (unsigned)(m < 0 ? -m : m);
  float y = (n % 2) ? x : 1.f;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.f / y : y;
}

// CIC deposit, cicpower.f90:76-98; returns rho_c(nw,nw,nw), x fastest.
template <class XT>
static void cic(const PGeo& G, const XT* xp, const int32_t* rhoc, int64_t nw, bool fixed, std::vector<float>& rho) {
  using U = typename std::make_unsigned<XT>::type;
  const int64_t nh = nw + 2;
  std::vector<float> halo;
  std::vector<int64_t> acc;
  if (fixed) acc.assign(nw * nw * nw, 0);
  else halo.assign(nh * nh * nh, 0.f);
  auto add = [&](int64_t ix, int64_t iy, int64_t iz, float w) {  // 1-based halo indices 0..nw+1
    if (fixed)
      acc[(wrap(iz - 1, nw) * nw + wrap(iy - 1, nw)) * nw + wrap(ix - 1, nw)] +=
          std::llrint(std::ldexp((double)w, 40));
    else
      halo[(iz * nh + iy) * nh + ix] += w;
  };
  int64_t ip = 0;
  const float fnw = (float)nw, fnc = (float)G.nc;
  for (int64_t tz = 0; tz < G.nnt; ++tz)
    for (int64_t ty = 0; ty < G.nnt; ++ty)
      for (int64_t tx = 0; tx < G.nnt; ++tx)
        for (int64_t k = 0; k < G.nt; ++k)
          for (int64_t j = 0; j < G.nt; ++j)
            for (int64_t i = 0; i < G.nt; ++i) {
              const int64_t s = ((((tz * G.nnt + ty) * G.nnt + tx) * G.nt + k) * G.nt + j) * G.nt + i;
              const int64_t g[3] = {tx * G.nt + i, ty * G.nt + j, tz * G.nt + k};
              for (int32_t l = 0; l < rhoc[s]; ++l, ++ip) {
                int64_t i1[3];
                float d1[3], d2[3];
                for (int d = 0; d < 3; ++d) {
                  // integer + real(8) decode, assigned to real(4) pos1
                  float pos = (float)((double)g[d] + ((double)(U)xp[3 * ip + d] + 0.5) * G.x_res);
                  pos = pos * fnw / fnc - 0.5f;
                  i1[d] = (int64_t)std::floor(pos) + 1;
                  d1[d] = (float)i1[d] - pos;
                  d2[d] = 1.f - d1[d];
                }
                const int64_t a = i1[0], b = i1[1], c = i1[2];
                add(a, b, c, d1[0] * d1[1] * d1[2]);
                add(a + 1, b, c, d2[0] * d1[1] * d1[2]);
                add(a, b + 1, c, d1[0] * d2[1] * d1[2]);
                add(a, b, c + 1, d1[0] * d1[1] * d2[2]);
                add(a, b + 1, c + 1, d1[0] * d2[1] * d2[2]);
                add(a + 1, b, c + 1, d2[0] * d1[1] * d2[2]);
                add(a + 1, b + 1, c, d2[0] * d2[1] * d1[2]);
                add(a + 1, b + 1, c + 1, d2[0] * d2[1] * d2[2]);
              }
            }
  rho.assign(nw * nw * nw, 0.f);
  if (fixed) {
    for (int64_t q = 0; q < nw * nw * nw; ++q) rho[q] = (float)std::ldexp((double)acc[q], -40);
    return;
  }
  auto H = [&](int64_t x, int64_t y, int64_t z) -> float& { return halo[(z * nh + y) * nh + x]; };
  // cicpower.f90:107-150 with nn=1: each face of the halo lands on the opposite interior layer
  for (int64_t z = 0; z < nh; ++z)
    for (int64_t y = 0; y < nh; ++y) H(1, y, z) += H(nw + 1, y, z);
  for (int64_t z = 0; z < nh; ++z)
    for (int64_t y = 0; y < nh; ++y) H(nw, y, z) += H(0, y, z);
  for (int64_t z = 0; z < nh; ++z)
    for (int64_t x = 0; x < nh; ++x) H(x, 1, z) += H(x, nw + 1, z);
  for (int64_t z = 0; z < nh; ++z)
    for (int64_t x = 0; x < nh; ++x) H(x, nw, z) += H(x, 0, z);
  for (int64_t y = 0; y < nh; ++y)
    for (int64_t x = 0; x < nh; ++x) H(x, y, 1) += H(x, y, nw + 1);
  for (int64_t y = 0; y < nh; ++y)
    for (int64_t x = 0; x < nh; ++x) H(x, y, nw) += H(x, y, 0);
  for (int64_t z = 1; z <= nw; ++z)
    for (int64_t y = 1; y <= nw; ++y)
      for (int64_t x = 1; x <= nw; ++x) rho[((z - 1) * nw + (y - 1)) * nw + (x - 1)] = H(x, y, z);
}

// interp1 (powerspectrum.f90:261-275).  auto_power passes the sections xi(2,:) and
// xi(5,:) of xi(10,0:nbin) to dummies of size nbin, so xdata(i) is bin i-1.
static float interp1(const float* xi, int64_t nbin, int row_x, int row_y, float xq) {
  auto X = [&](int64_t i) { return xi[(i - 1) * 10 + row_x]; };
  auto Y = [&](int64_t i) { return xi[(i - 1) * 10 + row_y]; };
  int64_t i1 = 1, i2 = nbin;
  while (i2 - i1 > 1) {
    const int64_t im = (i1 + i2) / 2;
    if (xq > X(im)) i1 = im;
    else i2 = im;
  }
  return Y(i1) + (xq - X(i1)) / (X(i2) - X(i1)) * (Y(i2) - Y(i1));
}

// pk_correction (powerspectrum.f90:212-259); returns alpha.
static float pk_correction(float* xi, int64_t nbin, int64_t nw, int p, int n_int) {
  const int64_t nyq = nw / 2;
  const float alpha = (std::log(interp1(xi, nbin, 1, 4, (float)nyq)) - std::log(interp1(xi, nbin, 1, 4, (float)nyq / 2))) /
                      std::log(2.f);
  if (std::isnan(alpha)) return alpha;
  std::vector<float> cd((nbin + 1) * 3, 0.f);
  const double PI = 4 * std::atan(1.0);
  for (int64_t i = 1; i <= nyq + 1; ++i)
    for (int64_t j = 1; j <= i; ++j)
      for (int64_t k = 1; k <= j; ++k) {
        const float kv[3] = {(float)(i - 1), (float)(j - 1), (float)(k - 1)};
        const float kmag = std::sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
        const int64_t ibin = std::lround(kmag);
        float w2p = 0.f;
        const float pk = std::pow(kmag, alpha);
        for (int in = -n_int; in <= n_int; ++in)
          for (int jn = -n_int; jn <= n_int; ++jn)
            for (int kn = -n_int; kn <= n_int; ++kn) {
              const float kn3[3] = {kv[0] + (float)(in * nw), kv[1] + (float)(jn * nw), kv[2] + (float)(kn * nw)};
              const float kmagn = std::sqrt(kn3[0] * kn3[0] + kn3[1] * kn3[1] + kn3[2] * kn3[2]);
              float prod = 1.f;
              for (int d = 0; d < 3; ++d) {
                const float ks = (float)(PI * (double)kn3[d] / (double)nw);
                prod = prod * (ks == 0.f ? 1.f : std::sin(ks) / ks);
              }
              w2p = w2p + powi(prod, 2 * p) * std::pow(kmagn, alpha);
            }
        cd[ibin * 3 + 0] += 1.f;
        cd[ibin * 3 + 1] += kmag;
        cd[ibin * 3 + 2] += w2p / pk;
      }
  for (int64_t b = 1; b <= nbin; ++b) {
    const float ratio = cd[b * 3 + 2] / cd[b * 3 + 0];
    xi[b * 10 + 4] = xi[b * 10 + 3] / ratio;
  }
  return alpha;
}

}  // namespace opower

extern "C" {

// xi: 10*(nbin+1) floats laid out as xi(10,0:nbin); delta: nw^3 floats or NULL.
// Returns nbin, or -1 on bad arguments.
int64_t oracle_power(const cube_params* p, const void* xp, const int32_t* rhoc, int64_t np, int64_t nw, int n_interp,
                     int n_int, int n_corr, int fixed, float* xi, float* delta, double* mean_out, float* alpha_out,
                     int* n_done) {
  using namespace opower;
  if (nw < 4 || nw % 2) return -1;
  const PGeo G = pgeo(p);
  std::vector<float> rho;
  if (G.izipx == 1) cic(G, (const int8_t*)xp, rhoc, nw, fixed != 0, rho);
  else cic(G, (const int16_t*)xp, rhoc, nw, fixed != 0, rho);
  const int64_t n3 = nw * nw * nw;
  double rho8 = 0;
  for (int64_t q = 0; q < n3; ++q) rho8 += (double)rho[q];
  const double mean = rho8 / (double)nw / (double)nw / (double)nw;
  for (int64_t q = 0; q < n3; ++q) rho[q] = (float)((double)rho[q] / mean - 1.0);
  if (delta) std::memcpy(delta, rho.data(), n3 * sizeof(float));
  // forward FFT, then cxyz/nw_global three times (powerspectrum.f90:150-151)
  std::vector<double> r(rho.begin(), rho.end());
  const int64_t nh = nw / 2 + 1;
  std::vector<std::complex<double>> ck(nw * nw * nh);
  oracle::rfft3<double>((int)nw, r.data(), ck.data());
  const int64_t nyq = nw / 2;
  const int64_t nbin = std::lround((float)nyq * std::sqrt(3.f));  // nint(nyquist*sqrt(3.))
  std::memset(xi, 0, 10 * (nbin + 1) * sizeof(float));
  const double PI = 4 * std::atan(1.0);
  const float fn = (float)nw, fnp = (float)np;
  for (int64_t k = 0; k < nw; ++k)
    for (int64_t j = 0; j < nw; ++j)
      for (int64_t i = 0; i <= nyq; ++i) {
        if (i == 0 && j == 0 && k == 0) continue;
        if ((i == 0 || i == nyq) && j > nyq) continue;
        if ((i == 0 || i == nyq) && (j == 0 || j == nyq) && k > nyq) continue;
        const int64_t m[3] = {i, j, k};
        float kx[3];
        for (int d = 0; d < 3; ++d) kx[d] = (float)(wrap(m[d] + nyq, nw) - nyq);
        const float kr = std::sqrt(kx[0] * kx[0] + kx[1] * kx[1] + kx[2] * kx[2]);
        const int64_t ibin = std::lround(kr);
        const std::complex<double> cv = ck[(k * nw + j) * nh + i];
        const float re = (float)cv.real() / fn / fn / fn, im = (float)cv.imag() / fn / fn / fn;
        const float amp = re * re + im * im;
        float c1k[3];
        for (int d = 0; d < 3; ++d) {
          const double s = std::sin(PI * (double)kx[d] / (double)nw);
          if (n_interp == 1) c1k[d] = 1.f;
          else if (n_interp == 2) c1k[d] = (float)(1.0 - (double)(2.f / 3.f) * (s * s));
          else c1k[d] = (float)(1.0 - s * s + (double)(2.f / 15.f) * ((s * s) * (s * s)));
        }
        const float dk = c1k[0] * c1k[1] * c1k[2] / fnp;
        float* x = xi + ibin * 10;
        x[0] += 1.f;
        x[1] += kr;
        x[2] += amp;
        x[3] += amp - dk;
      }
  for (int64_t b = 0; b <= nbin; ++b) {
    float* x = xi + b * 10;
    x[1] = x[1] / x[0];
    x[2] = x[2] / x[0];
    x[3] = x[3] / x[0];
    x[4] = x[3];
  }
  float alpha = 0.f;
  int done = 0;
  for (int it = 0; it < n_corr; ++it) {
    if (it > 0 && std::isnan(alpha)) break;
    alpha = pk_correction(xi, nbin, nw, n_interp, n_int);
    if (!std::isnan(alpha)) ++done;
  }
  const float box = p->box;
  const float box3 = powi(box, 3);
  for (int64_t b = 0; b <= nbin; ++b) {
    float* x = xi + b * 10;
    x[1] = (float)((double)x[1] * (2 * PI) / (double)box);
    x[2] = x[2] * box3;
    x[3] = x[3] * box3;
    x[4] = x[4] * box3;
  }
  if (mean_out) *mean_out = mean;
  if (alpha_out) *alpha_out = alpha;
  if (n_done) *n_done = done;
  return nbin;
}

}  // extern "C"
