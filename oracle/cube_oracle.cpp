// TEST INFRASTRUCTURE ONLY.
//
// CPU oracle: a restatement of CUBE's one-image (nn=1) P3M step, used by the tests as
// the checker for the CUDA path and by bench.py as the timed CPU baseline.  It is
// never linked into, loaded by, or called from the product library.
//
// Parity status: UNPINNED.  The reference is Coarray Fortran + FFTW and cannot be
// built here (no Fortran compiler, no FFTW), and its golden data
// (test/baseline.tar.gz) is a git-LFS pointer without payload.  This restatement
// follows the reference line by line (loop orders, FP32/FP64 kinds, integer
// wraps) and is pinned only by the reference's own runtime invariants (mass sums,
// count conservation, PID positivity, Green k=0) and by cross-checking the FFT
// against numpy.fft.
//
// Precision: T = float follows the reference's kinds (FP64 only where the
// reference uses real(8)); T = double is the FP64 oracle.  With nn=1 every ghost
// copy the reference makes (buffer_grid.f90, buffer_particle.f90) is a periodic
// image, so ghost cells are read through periodic indexing.
//
// Threading: boxes (tiles, subtiles) are independent in the reference (each kicks
// only its own physical particles), so OpenMP over boxes gives results identical
// to the serial order.

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <type_traits>
#include <vector>

#include "../include/cube_gpu.h"
#include "fft.hpp"

namespace oracle {

static const int RSF[8] = {0, 1, 2, 4, 6, 8, 12, 16};  // ratio_sf, parameters.f90:26 (1-based)

struct Geo {
  int64_t ng, rcs, nnt, nns, np_nc, ncb, ngb, nc, nt, ntt, ngp, ngt;
  int izipx;
  int64_t nfp[8], nfb[8], nft[8];
  float box, app, apm1c, apm2, apm3f, mass_p, f_nu;
  int pm3_on, pp_on;
  double x_res;
};

static Geo make_geo(const cube_params* p) {
  Geo g;
  g.ng = p->ng;
  g.rcs = p->ratio_cs;
  g.nnt = p->nnt;
  g.nns = p->nns;
  g.np_nc = p->np_nc;
  g.ncb = p->ncb;
  g.ngb = p->ngb;
  g.izipx = p->izipx;
  g.nc = g.ng / g.rcs;  // parameters.f90:57-62
  g.nt = g.nc / g.nnt;
  g.ntt = g.nt / g.nns;
  g.ngp = g.ng / g.nnt;
  g.ngt = g.ngp + 2 * g.ngb;
  for (int i = 1; i <= 7; ++i) {  // parameters.f90:66-69
    g.nfp[i] = (g.ngp / g.nns) * RSF[i];
    g.nfb[i] = g.rcs * RSF[i];
    g.nft[i] = g.nfp[i] + 2 * g.nfb[i];
  }
  g.nfp[0] = g.nfb[0] = g.nft[0] = 0;
  g.box = p->box;
  g.app = p->app;
  g.apm1c = p->apm1c;
  g.apm2 = p->apm2;
  g.apm3f = p->apm3f;
  g.mass_p = p->mass_p_cdm;
  g.f_nu = p->f_nu;
  g.pm3_on = p->pm3_on;
  g.pp_on = p->pp_on;
  g.x_res = std::ldexp(1.0, -8 * g.izipx);  // parameters.f90:132
  return g;
}

static inline int64_t wrapc(int64_t a, int64_t n) {
  a %= n;
  return a < 0 ? a + n : a;
}

// Index of global coarse cell (gx,gy,gz) (0-based, wrapped) in the reference's
// storage order rhoc(nt,nt,nt,nnt,nnt,nnt) (x fastest).
static inline int64_t cidx(const Geo& G, int64_t gx, int64_t gy, int64_t gz) {
  gx = wrapc(gx, G.nc);
  gy = wrapc(gy, G.nc);
  gz = wrapc(gz, G.nc);
  const int64_t tx = gx / G.nt, ty = gy / G.nt, tz = gz / G.nt;
  const int64_t lx = gx - tx * G.nt, ly = gy - ty * G.nt, lz = gz - tz * G.nt;
  return ((((tz * G.nnt + ty) * G.nnt + tx) * G.nt + lz) * G.nt + ly) * G.nt + lx;
}

// ZIPX decode: (int(xp+ishift,izipx)+rshift)*x_resolution (kick.f90:627-628) equals
// ((unsigned)xp + 0.5) * 2^(-8 izipx).
template <class XT>
static inline double zfrac(XT code, double x_res) {
  using U = typename std::make_unsigned<XT>::type;
  return ((double)(U)code + 0.5) * x_res;
}

struct Cells {
  const int32_t* rhoc;
  std::vector<int64_t> start;  // exclusive prefix in storage order
  Cells(const Geo& G, const int32_t* r) : rhoc(r) {
    const int64_t n = G.nc * G.nc * G.nc;
    start.resize(n + 1);
    start[0] = 0;
    for (int64_t i = 0; i < n; ++i) start[i + 1] = start[i] + r[i];
  }
};

// ---------------------------------------------------------------------------------
// Green's function, Green/Green.f90:1-80 (FP64; stored real32).  Table layout
// Gk(n/2+1, n, n), x fastest.
// ---------------------------------------------------------------------------------
static void green_3d(float* Gk, int64_t nglobal, float apm_soft, float apm_range, float gridsize) {
  const int64_t n1 = nglobal / 2 + 1, n2 = nglobal, n3 = nglobal;
  const float alpha = 4.f / 3;  // parameters.f90:53 (real4)
  const int p = 2, n_int = 2;
  std::vector<double> fftspace(nglobal);
  const float inv_n = 1.f / (float)nglobal;  // (1./nglobal) is default-real
  for (int64_t k = 1; k <= nglobal; ++k) {
    int64_t m = ((k + nglobal / 2 - 1) % nglobal) - nglobal / 2;
    fftspace[k - 1] = (2 * M_PI) * (double)inv_n * (double)m;
  }
  const double two15 = (double)(2.f / 15);
  const float gs2 = gridsize * gridsize;  // gridsize**(ndim-1), real4
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int64_t k3 = 0; k3 < n3; ++k3)
    for (int64_t k2 = 0; k2 < n2; ++k2)
      for (int64_t k1 = 0; k1 < n1; ++k1) {
        double kv[3] = {fftspace[k1], fftspace[k2], fftspace[k3]};
        double Dv[3], ur[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d)
          Dv[d] = (double)alpha * std::sin(kv[d]) + (double)(1 - alpha) * std::sin(2 * kv[d]) / 2;
        for (int i3 = -n_int; i3 <= n_int; ++i3)
          for (int i2 = -n_int; i2 <= n_int; ++i2)
            for (int i1 = -n_int; i1 <= n_int; ++i1) {
              double kn[3] = {kv[0] + 2 * M_PI * i1, kv[1] + 2 * M_PI * i2, kv[2] + 2 * M_PI * i3};
              double kmag = std::sqrt(kn[0] * kn[0] + kn[1] * kn[1] + kn[2] * kn[2]);
              double prod = 1;
              for (int d = 0; d < 3; ++d) prod *= (kn[d] == 0) ? 1.0 : std::sin(kn[d] / 2) / (kn[d] / 2);
              double Uk2 = std::pow(prod, 2 * p + 2);
              double Ss, Sr;
              double y = (double)apm_soft * kmag / 2;
              Ss = (kmag == 0) ? 1.0 : 12 * std::pow(y, -4) * (2 - 2 * std::cos(y) - y * std::sin(y));
              if (apm_range == 0) Sr = 0;
              else if (kmag == 0) Sr = 1;
              else {
                y = (double)apm_range * kmag / 2;
                Sr = 12 * std::pow(y, -4) * (2 - 2 * std::cos(y) - y * std::sin(y));
              }
              if (kmag == 0) continue;  // 0/0 only at k=0, which is zeroed below (Green.f90:71)
              for (int d = 0; d < 3; ++d) ur[d] += Uk2 * (kn[d] * (Ss * Ss - Sr * Sr) / (kmag * kmag));
            }
        double u2n = 1;
        for (int d = 0; d < 3; ++d) {
          double s = std::sin(kv[d] / 2);
          u2n *= 1 - s * s + two15 * s * s * s * s;
        }
        double num = Dv[0] * ur[0] + Dv[1] * ur[1] + Dv[2] * ur[2];
        double den = Dv[0] * Dv[0] + Dv[1] * Dv[1] + Dv[2] * Dv[2];
        double val = (den == 0) ? 0.0 : 4 * M_PI * num / den / (u2n * u2n) / (double)gs2;
        Gk[(k3 * n2 + k2) * n1 + k1] = (float)val;
      }
  // Gk(::nglobal/2,::nglobal/2,::nglobal/2)=0
  for (int64_t a = 0; a < n3; a += nglobal / 2)
    for (int64_t b = 0; b < n2; b += nglobal / 2)
      for (int64_t c = 0; c < n1; c += nglobal / 2) Gk[(a * n2 + b) * n1 + c] = 0;
}

// ---------------------------------------------------------------------------------
// drift.f90:1-233.  Outputs new particle arrays in the reference's order.
// ---------------------------------------------------------------------------------
template <class XT, class VT>
static int64_t drift_impl(const Geo& G, const XT* xp, const VT* vp, const int64_t* pid,
                          const int32_t* rhoc, float dt_old, float dt, float vz_max, XT* xo, VT* vo,
                          int64_t* po, int32_t* rhoc_o, int64_t tile_limit = -1) {
  Cells C(G, rhoc);
  const float dt_mid = (dt_old + dt) / 2;                  // drift.f90:21
  const int nlayer = 2 * (int)std::ceil(dt_mid * vz_max / (float)G.rcs) + 2;  // drift.f90:26
  const double inv = 1.0 / (G.x_res * (double)G.rcs);
  const int64_t nt = G.nt, ncb = G.ncb;
  const int64_t ntiles = (tile_limit > 0) ? std::min<int64_t>(tile_limit, G.nnt * G.nnt * G.nnt) : G.nnt * G.nnt * G.nnt;
  // per tile: destination lists (physical cells only)
  std::vector<int64_t> tile_count(ntiles, 0);
  std::vector<std::vector<std::vector<int64_t>>> dest(ntiles);
  int64_t err = 0;
#pragma omp parallel for schedule(dynamic) reduction(| : err)
  for (int64_t t = 0; t < ntiles; ++t) {
    const int64_t tx = t % G.nnt, ty = (t / G.nnt) % G.nnt, tz = t / (G.nnt * G.nnt);
    auto& D = dest[t];
    D.assign(nt * nt * nt, {});
    for (int il = 0; il < nlayer; ++il)
      for (int64_t k = 1 - ncb + il; k <= nt + ncb; k += nlayer)
        for (int64_t j = 1 - ncb; j <= nt + ncb; ++j)
          for (int64_t i = 1 - ncb; i <= nt + ncb; ++i) {
            const int64_t c = cidx(G, tx * nt + i - 1, ty * nt + j - 1, tz * nt + k - 1);
            const int64_t ijk[3] = {i, j, k};
            for (int64_t l = 0; l < rhoc[c]; ++l) {
              const int64_t ip = C.start[c] + l;
              int64_t ig[3];
              for (int d = 0; d < 3; ++d) {
                double deltax;
                if (std::is_same<VT, float>::value)
                  deltax = (double)((float)(dt_mid * (float)vp[3 * ip + d]) / (float)G.rcs);
                else
                  deltax = ((double)dt_mid * (double)vp[3 * ip + d]) / (double)G.rcs;
                const double xq = (double)(ijk[d] - 1) + zfrac<XT>(xp[3 * ip + d], G.x_res);
                ig[d] = (int64_t)std::ceil(xq + deltax);
              }
              const int64_t lo = 1 - 2 * ncb, hi = nt + 2 * ncb;
              if (ig[0] < lo || ig[1] < lo || ig[2] < lo || ig[0] > hi || ig[1] > hi || ig[2] > hi) {
                err |= 1;
                continue;
              }
              if (ig[0] >= 1 && ig[0] <= nt && ig[1] >= 1 && ig[1] <= nt && ig[2] >= 1 && ig[2] <= nt)
                D[((ig[2] - 1) * nt + (ig[1] - 1)) * nt + (ig[0] - 1)].push_back(ip);
            }
          }
    int64_t s = 0;
    for (auto& v : D) s += (int64_t)v.size();
    tile_count[t] = s;
  }
  if (err) return CUBE_E_RANGE;
  std::vector<int64_t> tile_off(ntiles + 1, 0);
  for (int64_t t = 0; t < ntiles; ++t) tile_off[t + 1] = tile_off[t] + tile_count[t];
#pragma omp parallel for schedule(dynamic)
  for (int64_t t = 0; t < ntiles; ++t) {
    int64_t o = tile_off[t];
    auto& D = dest[t];
    for (int64_t c = 0; c < nt * nt * nt; ++c) {
      rhoc_o[t * nt * nt * nt + c] = (int32_t)D[c].size();
      for (int64_t ip : D[c]) {
        for (int d = 0; d < 3; ++d) {
          int32_t dn;
          if (std::is_same<VT, float>::value)
            dn = (int32_t)std::llround((double)(float)(dt_mid * (float)vp[3 * ip + d]) * inv);
          else
            dn = (int32_t)std::llround((double)dt_mid * (double)vp[3 * ip + d] * inv);
          xo[3 * o + d] = (XT)(int32_t)((int32_t)xp[3 * ip + d] + dn);  // drift.f90:117, integer wrap
          vo[3 * o + d] = vp[3 * ip + d];
        }
        po[o] = pid[ip];
        ++o;
      }
    }
  }
  return tile_off[ntiles];
}

// ---------------------------------------------------------------------------------
// TSC weights (particle_mesh.f90:56-62, kick.f90:649-655), FP32 in the reference.
// ---------------------------------------------------------------------------------
template <class T>
static inline void tsc_w(double xpos, int64_t& i2, T w[3]) {
  const double fl = std::floor(xpos);
  i2 = (int64_t)fl + 1;
  const T l3 = (T)(xpos - fl);
  w[0] = (1 - l3) * (1 - l3) / 2;
  w[2] = l3 * l3 / 2;
  w[1] = 1 - w[0] - w[2];
}

// Fixed-point deposit: weight -> round(w * 2^40) as int64, summed exactly.
static const int FIXED_SHIFT = 40;

struct Box {
  int layer, iapm;
  int64_t tile[3];            // 0-based tile coords
  int64_t nc1[3], nc2[3];     // 1-based local coarse cell range of physical region
  int64_t nloop, nex, nphy, nwork, m1, m2, nforce, m1phi;
  float gridsize;
  int64_t ushift[3];          // utile_shift*nfp(iapm)
};

static Box make_pm2_box(const Geo& G, int64_t t) {
  Box b;
  b.layer = 2;
  b.iapm = 1;
  b.tile[0] = t % G.nnt;
  b.tile[1] = (t / G.nnt) % G.nnt;
  b.tile[2] = t / (G.nnt * G.nnt);
  for (int d = 0; d < 3; ++d) {  // kick.f90:54-58
    b.nc1[d] = 1;
    b.nc2[d] = G.nt;
    b.ushift[d] = 0;
  }
  b.nloop = G.ncb;
  b.nex = G.ngb + 1;
  b.nphy = G.ngp;
  b.nwork = G.ngt;
  b.m1 = 1 - G.ngb;
  b.m2 = G.ngp + G.ngb;
  b.nforce = G.ngp;
  b.m1phi = 1 - G.ngb;
  b.gridsize = 1.f;
  return b;
}

// Subtile numbering follows initialize.f90:351-367 (ixyz3): tile z,y,x outer, then
// subtile z,y,x.
static Box make_pm3_box(const Geo& G, int64_t s, int iapm) {
  Box b;
  const int64_t nns3 = G.nns * G.nns * G.nns;
  const int64_t t = s / nns3, f = s % nns3;
  b.layer = 3;
  b.iapm = iapm;
  b.tile[0] = t % G.nnt;
  b.tile[1] = (t / G.nnt) % G.nnt;
  b.tile[2] = t / (G.nnt * G.nnt);
  const int64_t us[3] = {f % G.nns, (f / G.nns) % G.nns, f / (G.nns * G.nns)};
  for (int d = 0; d < 3; ++d) {  // kick.f90:212-219
    b.nc1[d] = us[d] * G.ntt + 1;
    b.nc2[d] = (us[d] + 1) * G.ntt;
    b.ushift[d] = us[d] * G.nfp[iapm];
  }
  b.nloop = 1;
  b.nex = G.nfb[iapm] + 1;
  b.nphy = G.nfp[iapm];
  b.nwork = G.nft[iapm];
  b.m1 = 1 - G.nfb[iapm];
  b.m2 = G.nfp[iapm] + G.nfb[iapm];
  b.nforce = G.nfp[iapm];
  b.m1phi = 1 - G.nfb[iapm];
  b.gridsize = 1.f / (float)RSF[iapm];
  return b;
}

// Per-box work arrays.
template <class T>
struct BoxWork {
  std::vector<T> rho_th;                 // [1-nex, nphy+nex]^3
  std::vector<int64_t> rho_fx;           // fixed-point accumulator
  std::vector<T> dens;                   // nwork^3 (density, then phi)
  std::vector<std::complex<T>> ck;       // r2c output
  std::vector<T> force;                  // 3 x (nforce+2)^3
};

// Weighted gradient, parameters.f90:53-54 (real4 constants).
static const float W_ALPHA = 4.f / 3;
static const float WEIGHT[4] = {(W_ALPHA - 1) / 4, -W_ALPHA / 2, W_ALPHA / 2, (1 - W_ALPHA) / 4};

template <class T, class XT>
static void box_density(const Geo& G, const Cells& C, const XT* xp, const Box& b, BoxWork<T>& w,
                        bool fixed, int64_t& err, int64_t& mass_fx, double& mass_d) {
  const int64_t ne = b.nphy + 2 * b.nex;
  const int64_t o = 1 - b.nex;  // first index
  if (fixed) w.rho_fx.assign(ne * ne * ne, 0);
  else w.rho_th.assign(ne * ne * ne, (T)0);
  const double rcs = (double)G.rcs, gs = (double)b.gridsize;
  for (int il = 0; il < 3; ++il)  // nlayer=3 colouring (kick.f90:616-619)
    for (int64_t k = b.nc1[2] - b.nloop + il; k <= b.nc2[2] + b.nloop; k += 3)
      for (int64_t j = b.nc1[1] - b.nloop; j <= b.nc2[1] + b.nloop; ++j)
        for (int64_t i = b.nc1[0] - b.nloop; i <= b.nc2[0] + b.nloop; ++i) {
          const int64_t c = cidx(G, b.tile[0] * G.nt + i - 1, b.tile[1] * G.nt + j - 1, b.tile[2] * G.nt + k - 1);
          const int64_t ijk[3] = {i, j, k};
          for (int64_t l = 0; l < C.rhoc[c]; ++l) {
            const int64_t ip = C.start[c] + l;
            int64_t i2[3];
            T wt[3][3];
            for (int d = 0; d < 3; ++d) {
              double xpos = (double)(ijk[d] - 1) + zfrac<XT>(xp[3 * ip + d], G.x_res);
              xpos = xpos * rcs / gs - (double)b.ushift[d];  // kick.f90:628-629
              tsc_w<T>(xpos, i2[d], wt[d]);
              if (i2[d] - 1 < 1 - b.nex || i2[d] + 1 > b.nphy + b.nex) err |= 2;
            }
            if (err & 2) continue;
            for (int a3 = 0; a3 < 3; ++a3)
              for (int a2 = 0; a2 < 3; ++a2)
                for (int a1 = 0; a1 < 3; ++a1) {
                  const int64_t x = i2[0] - 1 + a1 - o, y = i2[1] - 1 + a2 - o, z = i2[2] - 1 + a3 - o;
                  const T ww = wt[0][a1] * wt[1][a2] * wt[2][a3];
                  if (fixed) w.rho_fx[(z * ne + y) * ne + x] += std::llrint(std::ldexp((double)(float)ww, FIXED_SHIFT));
                  else w.rho_th[(z * ne + y) * ne + x] += ww;
                }
          }
        }
  // ptotal = sum(1d0*rho_th(1:nphy,1:nphy,1:nphy))  (kick.f90:687-688)
  for (int64_t z = 1 - o; z <= b.nphy - o; ++z)
    for (int64_t y = 1 - o; y <= b.nphy - o; ++y)
      for (int64_t x = 1 - o; x <= b.nphy - o; ++x) {
        const int64_t s = (z * ne + y) * ne + x;
        if (fixed) mass_fx += w.rho_fx[s];
        else mass_d += (double)w.rho_th[s];
      }
  // density(nstart:nend) = rho_th(m1:m2)*mass_p_cdm  (kick.f90:686)
  const int64_t nw = b.nwork;
  w.dens.assign(nw * nw * nw, (T)0);
  for (int64_t z = 0; z < nw; ++z)
    for (int64_t y = 0; y < nw; ++y)
      for (int64_t x = 0; x < nw; ++x) {
        const int64_t s = ((z + b.m1 - o) * ne + (y + b.m1 - o)) * ne + (x + b.m1 - o);
        T r = fixed ? (T)(float)std::ldexp((double)w.rho_fx[s], -FIXED_SHIFT) : w.rho_th[s];
        w.dens[(z * nw + y) * nw + x] = r * (T)G.mass_p;
      }
}

// FFT, Green multiply, c2r and potential_to_force (kick.f90:697-716, 839-862).
template <class T>
static void box_force(const Box& b, const float* green, BoxWork<T>& w, T& f2max) {
  const int n = (int)b.nwork;
  const int nh = n / 2 + 1;
  w.ck.resize((int64_t)n * n * nh);
  rfft3<T>(n, w.dens.data(), w.ck.data());
  for (int64_t i = 0; i < (int64_t)n * n * nh; ++i) w.ck[i] *= (T)green[i];
  irfft3<T>(n, w.ck.data(), w.dens.data());
  const T norm = (T)((float)n * (float)n * (float)n);
  for (auto& v : w.dens) v = v / norm;  // phi=phi/(real(nwork)**3)
  const int64_t nf = b.nforce + 2;
  w.force.assign(3 * nf * nf * nf, (T)0);
  const int64_t off = -b.m1phi;  // phi index -> array index
  auto phi = [&](int64_t i, int64_t j, int64_t k) -> T {
    return w.dens[((k + off) * n + (j + off)) * n + (i + off)];
  };
  T fm = 0;
  for (int64_t k = 0; k < nf; ++k)
    for (int64_t j = 0; j < nf; ++j)
      for (int64_t i = 0; i < nf; ++i) {
        T f[3] = {0, 0, 0};
        const int sh[4] = {-2, -1, 1, 2};
        for (int q = 0; q < 4; ++q) f[0] += phi(i + sh[q], j, k) * (T)WEIGHT[q];
        for (int q = 0; q < 4; ++q) f[1] += phi(i, j + sh[q], k) * (T)WEIGHT[q];
        for (int q = 0; q < 4; ++q) f[2] += phi(i, j, k + sh[q]) * (T)WEIGHT[q];
        for (int d = 0; d < 3; ++d) w.force[((k * nf + j) * nf + i) * 3 + d] = f[d];
        if (i >= 1 && i <= b.nforce && j >= 1 && j <= b.nforce && k >= 1 && k <= b.nforce) {
          T s = f[0] * f[0] + f[1] * f[1] + f[2] * f[2];
          fm = std::max(fm, s);
        }
      }
  f2max = fm;
}

// vp += dv*a_mid*dt/6/pi  (kick.f90:797; the last division is by real(8) pi).
template <class T>
static inline T kick_add(T v, T dv, float a_mid, float dt) {
  if (std::is_same<T, float>::value) {
    float t = (float)dv * a_mid * dt / 6;
    return (T)(float)((double)(float)v + (double)t / M_PI);
  } else {
    return v + dv * (double)a_mid * (double)dt / 6 / M_PI;
  }
}

template <class T, class XT>
static void box_interp(const Geo& G, const Cells& C, const XT* xp, T* vp, const Box& b, const BoxWork<T>& w,
                       float a_mid, float dt, T vmax[3], int64_t& err) {
  const int64_t nf = b.nforce + 2;
  const double rcs = (double)G.rcs, gs = (double)b.gridsize;
  for (int64_t k = b.nc1[2]; k <= b.nc2[2]; ++k)
    for (int64_t j = b.nc1[1]; j <= b.nc2[1]; ++j)
      for (int64_t i = b.nc1[0]; i <= b.nc2[0]; ++i) {
        const int64_t c = cidx(G, b.tile[0] * G.nt + i - 1, b.tile[1] * G.nt + j - 1, b.tile[2] * G.nt + k - 1);
        const int64_t ijk[3] = {i, j, k};
        for (int64_t l = 0; l < C.rhoc[c]; ++l) {
          const int64_t ip = C.start[c] + l;
          int64_t i2[3];
          T wt[3][3];
          for (int d = 0; d < 3; ++d) {
            double xpos = (double)(ijk[d] - 1) + zfrac<XT>(xp[3 * ip + d], G.x_res);
            xpos = xpos * rcs / gs - (double)b.ushift[d];
            tsc_w<T>(xpos, i2[d], wt[d]);
            if (i2[d] - 1 < 0 || i2[d] + 1 > b.nforce + 1) err |= 4;
          }
          if (err & 4) continue;
          T dv[3] = {0, 0, 0};
          for (int a3 = 0; a3 < 3; ++a3)
            for (int a2 = 0; a2 < 3; ++a2)
              for (int a1 = 0; a1 < 3; ++a1) {
                const int64_t x = i2[0] - 1 + a1, y = i2[1] - 1 + a2, z = i2[2] - 1 + a3;
                const T* F = &w.force[((z * nf + y) * nf + x) * 3];
                for (int d = 0; d < 3; ++d) dv[d] = dv[d] + F[d] * wt[0][a1] * wt[1][a2] * wt[2][a3];
              }
          for (int d = 0; d < 3; ++d) {
            vp[3 * ip + d] = kick_add<T>(vp[3 * ip + d], dv[d], a_mid, dt);
            vmax[d] = std::max(vmax[d], (T)std::fabs(vp[3 * ip + d]));
          }
        }
      }
}

// ---------------------------------------------------------------------------------
// PM1, particle_mesh.f90:1-222: global periodic nc^3 mesh.
// ---------------------------------------------------------------------------------
template <class T, class XT>
static void pm1(const Geo& G, const Cells& C, const XT* xp, T* vp, const float* green, bool fixed, float a_mid,
                float dt, T& f2max, std::vector<T>* dbg_dens, std::vector<T>* dbg_phi, std::vector<T>* dbg_force,
                int64_t& err, double& mass) {
  const int64_t nc = G.nc, nt = G.nt;
  std::vector<T> rho(nc * nc * nc, (T)0);
  const int64_t ntiles = G.nnt * G.nnt * G.nnt;
  const int64_t nex = 2, ne = nt + 2 * nex;
  int64_t e = 0, mfx = 0;
  double md = 0.0;
#pragma omp parallel for schedule(dynamic) reduction(| : e) reduction(+ : mfx, md)
  for (int64_t t = 0; t < ntiles; ++t) {
    const int64_t tx = t % G.nnt, ty = (t / G.nnt) % G.nnt, tz = t / (G.nnt * G.nnt);
    std::vector<T> rex;
    std::vector<int64_t> rfx;
    if (fixed) rfx.assign(ne * ne * ne, 0);
    else rex.assign(ne * ne * ne, (T)0);
    for (int il = 0; il < 3; ++il)
      for (int64_t k = 0 + il; k <= nt + 1; k += 3)
        for (int64_t j = 0; j <= nt + 1; ++j)
          for (int64_t i = 0; i <= nt + 1; ++i) {
            const int64_t c = cidx(G, tx * nt + i - 1, ty * nt + j - 1, tz * nt + k - 1);
            const int64_t ijk[3] = {i, j, k};
            for (int64_t l = 0; l < C.rhoc[c]; ++l) {
              const int64_t ip = C.start[c] + l;
              int64_t i2[3];
              T wt[3][3];
              for (int d = 0; d < 3; ++d) {
                double xpos = (double)(ijk[d] - 1) + zfrac<XT>(xp[3 * ip + d], G.x_res);
                xpos = xpos * (double)G.rcs / (double)(float)G.rcs;
                tsc_w<T>(xpos, i2[d], wt[d]);
                if (i2[d] - 1 < 1 - nex || i2[d] + 1 > nt + nex) e |= 2;
              }
              if (e & 2) continue;
              for (int a3 = 0; a3 < 3; ++a3)
                for (int a2 = 0; a2 < 3; ++a2)
                  for (int a1 = 0; a1 < 3; ++a1) {
                    const int64_t x = i2[0] - 1 + a1 - (1 - nex), y = i2[1] - 1 + a2 - (1 - nex),
                                  z = i2[2] - 1 + a3 - (1 - nex);
                    const T ww = wt[0][a1] * wt[1][a2] * wt[2][a3];
                    if (fixed) rfx[(z * ne + y) * ne + x] += std::llrint(std::ldexp((double)(float)ww, FIXED_SHIFT));
                    else rex[(z * ne + y) * ne + x] += ww;
                  }
            }
          }
    for (int64_t k = 1; k <= nt; ++k)
      for (int64_t j = 1; j <= nt; ++j)
        for (int64_t i = 1; i <= nt; ++i) {
          const int64_t s = ((k - 1 + nex) * ne + (j - 1 + nex)) * ne + (i - 1 + nex);
          T r = fixed ? (T)(float)std::ldexp((double)rfx[s], -FIXED_SHIFT) : rex[s];
          rho[((tz * nt + k - 1) * nc + (ty * nt + j - 1)) * nc + (tx * nt + i - 1)] = r * (T)G.mass_p;
          // testrho = testrho + sum(1d0*rho_ex(1:nphy,1:nphy,1:nphy))  (particle_mesh.f90:106)
          if (fixed) mfx += rfx[s];
          else md += (double)rex[s];
        }
  }
  err |= e;
  mass = fixed ? std::ldexp((double)mfx, -FIXED_SHIFT) : md;
  if (dbg_dens) *dbg_dens = rho;
  const int n = (int)nc, nh = n / 2 + 1;
  std::vector<std::complex<T>> ck((int64_t)n * n * nh);
  rfft3<T>(n, rho.data(), ck.data());
  for (int64_t i = 0; i < (int64_t)n * n * nh; ++i) ck[i] *= (T)green[i];
  irfft3<T>(n, ck.data(), rho.data());
  for (auto& v : rho) v = v / (T)(float)nc / (T)(float)nc / (T)(float)nc;  // pencil_fft.f90:77
  if (dbg_phi) *dbg_phi = rho;
  // grad with 3-cell periodic halo (particle_mesh.f90:136-141, 224-247)
  const int64_t nf = nc + 2;
  std::vector<T> force(3 * nf * nf * nf);
  auto phi = [&](int64_t i, int64_t j, int64_t k) -> T {
    return rho[(wrapc(k - 1, nc) * nc + wrapc(j - 1, nc)) * nc + wrapc(i - 1, nc)];
  };
  T fm = 0;
  const int sh[4] = {-2, -1, 1, 2};
  for (int64_t k = 0; k < nf; ++k)
    for (int64_t j = 0; j < nf; ++j)
      for (int64_t i = 0; i < nf; ++i) {
        T f[3] = {0, 0, 0};
        for (int q = 0; q < 4; ++q) f[0] += phi(i + sh[q], j, k) * (T)WEIGHT[q];
        for (int q = 0; q < 4; ++q) f[1] += phi(i, j + sh[q], k) * (T)WEIGHT[q];
        for (int q = 0; q < 4; ++q) f[2] += phi(i, j, k + sh[q]) * (T)WEIGHT[q];
        for (int d = 0; d < 3; ++d) force[((k * nf + j) * nf + i) * 3 + d] = f[d];
        if (i >= 1 && i <= nc && j >= 1 && j <= nc && k >= 1 && k <= nc)
          fm = std::max(fm, f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
      }
  f2max = fm;
  if (dbg_force) *dbg_force = force;
  // interpolation and kick (particle_mesh.f90:148-217)
#pragma omp parallel for schedule(dynamic) reduction(| : e)
  for (int64_t t = 0; t < ntiles; ++t) {
    const int64_t tx = t % G.nnt, ty = (t / G.nnt) % G.nnt, tz = t / (G.nnt * G.nnt);
    for (int64_t k = 1; k <= nt; ++k)
      for (int64_t j = 1; j <= nt; ++j)
        for (int64_t i = 1; i <= nt; ++i) {
          const int64_t c = cidx(G, tx * nt + i - 1, ty * nt + j - 1, tz * nt + k - 1);
          const int64_t g[3] = {tx * nt + i, ty * nt + j, tz * nt + k};
          for (int64_t l = 0; l < C.rhoc[c]; ++l) {
            const int64_t ip = C.start[c] + l;
            int64_t i2[3];
            T wt[3][3];
            for (int d = 0; d < 3; ++d) {
              double xpos = (double)(g[d] - 1) + zfrac<XT>(xp[3 * ip + d], G.x_res);
              xpos = xpos * (double)G.rcs / (double)(float)G.rcs;
              tsc_w<T>(xpos, i2[d], wt[d]);
            }
            T dv[3] = {0, 0, 0};
            for (int a3 = 0; a3 < 3; ++a3)
              for (int a2 = 0; a2 < 3; ++a2)
                for (int a1 = 0; a1 < 3; ++a1) {
                  const int64_t x = i2[0] - 1 + a1, y = i2[1] - 1 + a2, z = i2[2] - 1 + a3;
                  const T* F = &force[((z * nf + y) * nf + x) * 3];
                  for (int d = 0; d < 3; ++d) dv[d] = dv[d] + F[d] * wt[0][a1] * wt[1][a2] * wt[2][a3];
                }
            for (int d = 0; d < 3; ++d) vp[3 * ip + d] = kick_add<T>(vp[3 * ip + d], dv[d], a_mid, dt);
          }
        }
  }
  err |= e;
}

// ---------------------------------------------------------------------------------
// PP, kick.f90:360-588.
// ---------------------------------------------------------------------------------
template <class T>
static inline T F_ra(T r, T apm) {
  T ep = 2 * r / apm;
  if (apm == 0 || ep > 2) return 1 / (r * r);
  const T c = (T)1 / (T)35 / (apm * apm);
  T e2 = ep * ep, e3 = e2 * ep, e4 = e3 * ep, e5 = e4 * ep, e6 = e5 * ep;
  if (ep > 1) return c * (12 * (1 / e2) - 224 + 896 * ep - 840 * e2 + 224 * e3 + 70 * e4 - 48 * e5 + 7 * e6);
  if (ep > 0) return c * (224 * ep - 224 * e3 + 70 * e4 + 48 * e5 - 21 * e6);
  return 0;
}

static const int NEIGH[13][3] = {  // initialize.f90:369-390
    {-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {-1, 0, -1}, {0, 0, -1}, {1, 0, -1}, {-1, 1, -1},
    {0, 1, -1},   {1, 1, -1},  {-1, -1, 0}, {0, -1, 0},  {1, -1, 0}, {-1, 0, 0}};

template <class T, class XT>
static void pp_box(const Geo& G, const Cells& C, const XT* xp, T* vp, const Box& b, float a_mid, float dt,
                   T& f2max_t, T vmax_t[3], int64_t& npairs, int64_t& err) {
  const int rcp = RSF[b.iapm];
  const int64_t npgrid = G.ntt * rcp;
  const float pp_range_f = 3.5f / (float)rcp;  // apm3(iapm), parameters.f90:43
  const T pp_range = (T)pp_range_f, pp_range2 = pp_range * pp_range;
  const T app = (T)G.app;
  const int64_t ng2 = npgrid + 2;
  std::vector<int32_t> cell_count(ng2 * ng2 * ng2, 0), cell_start(ng2 * ng2 * ng2, 0), cell_off(ng2 * ng2 * ng2, 0);
  auto ci = [&](int64_t i, int64_t j, int64_t k) { return (k * ng2 + j) * ng2 + i; };
  std::vector<int64_t> pcell, ip_tmp;
  std::vector<T> xf_tmp;
  int64_t n_phy = 0, n_ext = 0;
  const int64_t us[3] = {(b.nc1[0] - 1) / G.ntt, (b.nc1[1] - 1) / G.ntt, (b.nc1[2] - 1) / G.ntt};
  // Pass 1 (kick.f90:412-459)
  for (int64_t k = b.nc1[2] - 1; k <= b.nc2[2] + 1; ++k)
    for (int64_t j = b.nc1[1] - 1; j <= b.nc2[1] + 1; ++j)
      for (int64_t i = b.nc1[0] - 1; i <= b.nc2[0] + 1; ++i) {
        const int64_t c = cidx(G, b.tile[0] * G.nt + i - 1, b.tile[1] * G.nt + j - 1, b.tile[2] * G.nt + k - 1);
        const int64_t ijk[3] = {i, j, k};
        for (int64_t l = 0; l < C.rhoc[c]; ++l) {
          const int64_t ip = C.start[c] + l;
          ip_tmp.push_back(ip);
          int64_t idx[3];
          for (int d = 0; d < 3; ++d) {
            float xv = (float)((double)(ijk[d] - 1) + zfrac<XT>(xp[3 * ip + d], G.x_res));  // real4 xvec
            xf_tmp.push_back((T)(xv * (float)G.rcs));
            float xr = (float)rcp * (xv - (float)(us[d] * G.ntt));
            idx[d] = (int64_t)std::floor(xr) + 1;
            if (idx[d] < 1 - rcp || idx[d] > npgrid + rcp) err |= 8;
          }
          if (idx[0] >= 0 && idx[1] >= 0 && idx[2] >= 0 && idx[0] <= npgrid + 1 && idx[1] <= npgrid + 1 &&
              idx[2] <= npgrid + 1) {
            pcell.push_back(ci(idx[0], idx[1], idx[2]));
            cell_count[pcell.back()]++;
            ++n_ext;
            if (idx[0] >= 1 && idx[1] >= 1 && idx[2] >= 1 && idx[0] <= npgrid && idx[1] <= npgrid && idx[2] <= npgrid)
              ++n_phy;
          } else {
            pcell.push_back(-1);
          }
        }
      }
  if (ip_tmp.empty()) return;
  // Pass 2 (kick.f90:468-499)
  std::vector<int64_t> act, act_ext;
  int32_t pos = 0;
  for (int64_t k = 1; k <= npgrid; ++k)
    for (int64_t j = 1; j <= npgrid; ++j)
      for (int64_t i = 1; i <= npgrid; ++i) {
        const int64_t c = ci(i, j, k);
        cell_start[c] = cell_off[c] = pos;
        pos += cell_count[c];
        if (cell_count[c] > 0) act.push_back(c);
      }
  for (int64_t k = 0; k <= npgrid + 1; ++k)
    for (int64_t j = 0; j <= npgrid + 1; ++j)
      for (int64_t i = 0; i <= npgrid + 1; ++i) {
        const int64_t c = ci(i, j, k);
        if (cell_count[c] > 0) act_ext.push_back(c);
        if (i >= 1 && i <= npgrid && j >= 1 && j <= npgrid && k >= 1 && k <= npgrid) continue;
        cell_start[c] = cell_off[c] = pos;
        pos += cell_count[c];
      }
  // Pass 3
  std::vector<T> xf(3 * std::max<int64_t>(1, n_ext)), af(3 * std::max<int64_t>(1, n_ext), (T)0);
  std::vector<int64_t> ip_local(std::max<int64_t>(1, n_phy));
  for (size_t l = 0; l < pcell.size(); ++l)
    if (pcell[l] >= 0) {
      const int32_t p = cell_off[pcell[l]]++;
      for (int d = 0; d < 3; ++d) xf[3 * p + d] = xf_tmp[3 * l + d];
      if (p < n_phy) ip_local[p] = ip_tmp[l];
    }
  int64_t np_ = 0;
  auto pair = [&](int64_t p1, int64_t p2, T* f1, bool self) {
    T rv[3] = {xf[3 * p2] - xf[3 * p1], xf[3 * p2 + 1] - xf[3 * p1 + 1], xf[3 * p2 + 2] - xf[3 * p1 + 2]};
    T r2 = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    if ((self ? (r2 > 0) : true) && r2 < pp_range2) {
      T rm = std::sqrt(r2);
      T s = F_ra<T>(rm, app) - F_ra<T>(rm, pp_range);
      for (int d = 0; d < 3; ++d) {
        T fpp = rv[d] / rm * s;
        f1[d] += fpp;
        af[3 * p2 + d] -= fpp;
      }
      ++np_;
    }
  };
  // self (kick.f90:516-534)
  for (int64_t c : act) {
    const int64_t s1 = cell_start[c], e1 = s1 + cell_count[c] - 1;
    for (int64_t p1 = s1; p1 < e1; ++p1) {
      T f1[3] = {af[3 * p1], af[3 * p1 + 1], af[3 * p1 + 2]};
      for (int64_t p2 = p1 + 1; p2 <= e1; ++p2) pair(p1, p2, f1, true);
      for (int d = 0; d < 3; ++d) af[3 * p1 + d] = f1[d];
    }
  }
  // neighbours (kick.f90:537-566)
  for (int64_t c : act_ext) {
    const int64_t i = c % ng2, j = (c / ng2) % ng2, k = c / (ng2 * ng2);
    const int64_t s1 = cell_start[c], e1 = s1 + cell_count[c] - 1;
    const bool ghost = (std::min({i, j, k}) == 0 || std::max({i, j, k}) == npgrid + 1);
    for (int n = 0; n < 13; ++n) {
      const int64_t a = i + NEIGH[n][0], bb = j + NEIGH[n][1], cc = k + NEIGH[n][2];
      if (std::min({a, bb, cc}) < 0 || std::max({a, bb, cc}) > npgrid + 1) continue;
      if (ghost && (std::min({a, bb, cc}) == 0 || std::max({a, bb, cc}) == npgrid + 1)) continue;
      const int64_t c2 = ci(a, bb, cc);
      if (cell_count[c2] == 0) continue;
      const int64_t s2 = cell_start[c2], e2 = s2 + cell_count[c2] - 1;
      for (int64_t p1 = s1; p1 <= e1; ++p1) {
        T f1[3] = {af[3 * p1], af[3 * p1 + 1], af[3 * p1 + 2]};
        for (int64_t p2 = s2; p2 <= e2; ++p2) pair(p1, p2, f1, false);
        for (int d = 0; d < 3; ++d) af[3 * p1 + d] = f1[d];
      }
    }
  }
  // kick (kick.f90:569-582)
  T mass_scale, v_scale;
  if (std::is_same<T, float>::value) {
    mass_scale = (G.f_nu > 0) ? (T)(float)((double)G.mass_p * ((1 - (double)G.f_nu) * (1 - (double)G.f_nu)))
                              : (T)G.mass_p;
    v_scale = (T)(float)((double)(a_mid * dt / 6) / M_PI);
  } else {
    mass_scale = (T)G.mass_p * ((G.f_nu > 0) ? (1 - (T)G.f_nu) * (1 - (T)G.f_nu) : (T)1);
    v_scale = (T)a_mid * (T)dt / 6 / M_PI;
  }
  for (int64_t p = 0; p < n_phy; ++p) {
    T f1[3];
    for (int d = 0; d < 3; ++d) f1[d] = af[3 * p + d] * mass_scale;
    f2max_t = std::max(f2max_t, f1[0] * f1[0] + f1[1] * f1[1] + f1[2] * f1[2]);
    const int64_t ip = ip_local[p];
    for (int d = 0; d < 3; ++d) {
      vp[3 * ip + d] = vp[3 * ip + d] + f1[d] * v_scale;
      vmax_t[d] = std::max(vmax_t[d], (T)std::fabs(vp[3 * ip + d]));
    }
  }
  npairs += np_;
}

// Subtile class from the largest coarse-cell count (kick.f90:108-133).
static void classify(const Geo& G, const int32_t* rhoc, std::vector<int>& ires, int32_t napm[8]) {
  const int64_t nns3 = G.nns * G.nns * G.nns, ns3 = G.nnt * G.nnt * G.nnt * nns3;
  ires.assign(ns3, 2);
  for (int i = 0; i < 8; ++i) napm[i] = 0;
  for (int64_t s = 0; s < ns3; ++s) {
    Box b = make_pm3_box(G, s, 2);
    int32_t mx = 0;
    for (int64_t k = b.nc1[2]; k <= b.nc2[2]; ++k)
      for (int64_t j = b.nc1[1]; j <= b.nc2[1]; ++j)
        for (int64_t i = b.nc1[0]; i <= b.nc2[0]; ++i)
          mx = std::max(mx, rhoc[cidx(G, b.tile[0] * G.nt + i - 1, b.tile[1] * G.nt + j - 1, b.tile[2] * G.nt + k - 1)]);
    const float npc = (float)mx / 64.f;
    int r = (npc < 24) ? 2 : (npc < 114) ? 3 : (npc < 320) ? 4 : 5;
    ires[s] = r;
    napm[r]++;
  }
}

static inline float dt_crit(float coef, float f2max, float a_mid) {
  const float G_grid = (float)((double)(1.0f / 6.0f) / M_PI);  // variables.f90:28
  return coef * std::sqrt(1.f / (std::sqrt(f2max) * a_mid * G_grid));
}

}  // namespace oracle

using namespace oracle;

extern "C" {

typedef struct oracle_kick_out {
  double t_pm1, t_pm2, t_pm3, t_pp;  // wall seconds per stage
  double f2max_pm1, f2max_pm2, f2max_pm3, f2max_pp;
  double vmax[3];
  float dt_pm1, dt_pm2, dt_pm3, dt_pp, dt_vmax, vz_max;
  int32_t napm[8];
  int64_t pp_pairs;
  int64_t err;
  // sum of the density over each level's physical cells, particle units (particle_mesh.f90:106
  // testrho, kick.f90:687-688 ptotal): exact int64 sums with the fixed-point deposit
  double mass[3];
} oracle_kick_out;

int oracle_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// Green table of level 1 (PM1), 2 (PM2) or 3 (PM3 class iapm), initialize.f90:247-284.
int oracle_green(const cube_params* p, int level, int iapm, float* out) {
  Geo G = make_geo(p);
  if (level == 1) green_3d(out, G.nc, G.apm1c, 0.f, (float)G.rcs);
  else if (level == 2) green_3d(out, G.ngt, G.apm2, G.apm1c * (float)G.rcs, 1.f);
  else if (level == 3) {
    if (iapm < 2 || iapm > 5) return CUBE_E_ARG;
    green_3d(out, G.nft[iapm], G.apm3f, G.apm2 * (float)RSF[iapm], 1.f / (float)RSF[iapm]);
  } else return CUBE_E_ARG;
  return 0;
}

// FFT self-test helpers: 3D r2c forward / c2r backward (unnormalised).
int oracle_rfft3(int n, const double* r, double* c_interleaved) {
  rfft3<double>(n, r, reinterpret_cast<std::complex<double>*>(c_interleaved));
  return 0;
}
int oracle_irfft3(int n, double* c_interleaved, double* r) {
  irfft3<double>(n, reinterpret_cast<std::complex<double>*>(c_interleaved), r);
  return 0;
}

// drift.f90, FP32 velocities. Returns the new particle count or a negative code.
int64_t oracle_drift(const cube_params* p, const void* xp, const float* vp, const int64_t* pid, const int32_t* rhoc,
                     float dt_old, float dt, float vz_max, void* xo, float* vo, int64_t* po, int32_t* rhoc_o) {
  Geo G = make_geo(p);
  if (G.izipx == 1)
    return drift_impl<int8_t, float>(G, (const int8_t*)xp, vp, pid, rhoc, dt_old, dt, vz_max, (int8_t*)xo, vo, po, rhoc_o);
  return drift_impl<int16_t, float>(G, (const int16_t*)xp, vp, pid, rhoc, dt_old, dt, vz_max, (int16_t*)xo, vo, po, rhoc_o);
}
// drift.f90 restricted to the first `tiles` tiles (CPU-baseline timing sample): returns
// the number of particles those tiles receive.
int64_t oracle_drift_sample(const cube_params* p, const void* xp, const float* vp, const int64_t* pid,
                            const int32_t* rhoc, float dt_old, float dt, float vz_max, void* xo, float* vo, int64_t* po,
                            int32_t* rhoc_o, int64_t tiles) {
  Geo G = make_geo(p);
  if (G.izipx == 1)
    return drift_impl<int8_t, float>(G, (const int8_t*)xp, vp, pid, rhoc, dt_old, dt, vz_max, (int8_t*)xo, vo, po, rhoc_o,
                                     tiles);
  return drift_impl<int16_t, float>(G, (const int16_t*)xp, vp, pid, rhoc, dt_old, dt, vz_max, (int16_t*)xo, vo, po,
                                    rhoc_o, tiles);
}

int64_t oracle_drift64(const cube_params* p, const void* xp, const double* vp, const int64_t* pid, const int32_t* rhoc,
                       float dt_old, float dt, float vz_max, void* xo, double* vo, int64_t* po, int32_t* rhoc_o) {
  Geo G = make_geo(p);
  if (G.izipx == 1)
    return drift_impl<int8_t, double>(G, (const int8_t*)xp, vp, pid, rhoc, dt_old, dt, vz_max, (int8_t*)xo, vo, po, rhoc_o);
  return drift_impl<int16_t, double>(G, (const int16_t*)xp, vp, pid, rhoc, dt_old, dt, vz_max, (int16_t*)xo, vo, po, rhoc_o);
}

}  // extern "C"

namespace oracle {

// Full kick (kick.f90:1-353).  `only` selects levels (bitmask 1 PM1, 2 PM2, 4 PM3,
// 8 PP) so tests can isolate one level; the reference order is always kept.
// `boxes_frac` > 0 limits PM2/PM3/PP to the first fraction of boxes (CPU baseline
// sampling only).
template <class T, class XT>
static int kick_impl(const Geo& G, const XT* xp, T* vp, const int32_t* rhoc, float dt, float a_mid, bool fixed,
                     int only, double boxes_frac, oracle_kick_out* out, int dbg_level, int64_t dbg_box, int dbg_what,
                     float* dbg_out, int64_t dbg_n) {
  Cells C(G, rhoc);
  int64_t err = 0;
  std::memset(out, 0, sizeof(*out));
  std::vector<float> g1(G.nc * G.nc * (G.nc / 2 + 1));
  green_3d(g1.data(), G.nc, G.apm1c, 0.f, (float)G.rcs);
  auto dump = [&](const std::vector<T>& v) {
    if (!dbg_out) return;
    int64_t n = std::min<int64_t>(dbg_n, (int64_t)v.size());
    for (int64_t i = 0; i < n; ++i) dbg_out[i] = (float)v[i];
  };
  T vmax[3] = {0, 0, 0};
  double t0 = omp_get_wtime();
  // PM1
  T f2 = 0;
  if (only & 1) {
    std::vector<T> dd, dp, df;
    const bool want = dbg_level == 1;
    pm1<T, XT>(G, C, xp, vp, g1.data(), fixed, a_mid, dt, f2, want && dbg_what == 0 ? &dd : nullptr,
               want && dbg_what == 1 ? &dp : nullptr, want && dbg_what == 2 ? &df : nullptr, err, out->mass[0]);
    if (want) dump(dbg_what == 0 ? dd : dbg_what == 1 ? dp : df);
  }
  out->f2max_pm1 = (double)f2;
  out->dt_pm1 = dt_crit(0.5f, (float)f2, a_mid);
  out->t_pm1 = omp_get_wtime() - t0;
  t0 = omp_get_wtime();
  // PM2
  const int64_t ntiles = G.nnt * G.nnt * G.nnt;
  const int64_t ntile_run = boxes_frac > 0 ? std::max<int64_t>(1, (int64_t)(ntiles * boxes_frac)) : ntiles;
  if (only & 2) {
    std::vector<float> g2(G.ngt * G.ngt * (G.ngt / 2 + 1));
    green_3d(g2.data(), G.ngt, G.apm2, G.apm1c * (float)G.rcs, 1.f);
    T f2m = 0, vm0 = 0, vm1 = 0, vm2 = 0;
    int64_t e = 0, mfx = 0;
    double md = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : f2m, vm0, vm1, vm2) reduction(| : e) reduction(+ : mfx, md)
    for (int64_t t = 0; t < ntile_run; ++t) {
      BoxWork<T> w;
      Box b = make_pm2_box(G, t);
      box_density<T, XT>(G, C, xp, b, w, fixed, e, mfx, md);
      if (dbg_level == 2 && dbg_box == t && dbg_what == 0) dump(w.dens);
      T f2t = 0;
      box_force<T>(b, g2.data(), w, f2t);
      if (dbg_level == 2 && dbg_box == t && dbg_what == 1) dump(w.dens);
      if (dbg_level == 2 && dbg_box == t && dbg_what == 2) dump(w.force);
      T vm[3] = {0, 0, 0};
      box_interp<T, XT>(G, C, xp, vp, b, w, a_mid, dt, vm, e);
      f2m = std::max(f2m, f2t);
      vm0 = std::max(vm0, vm[0]);
      vm1 = std::max(vm1, vm[1]);
      vm2 = std::max(vm2, vm[2]);
    }
    err |= e;
    out->mass[1] = fixed ? std::ldexp((double)mfx, -FIXED_SHIFT) : md;
    out->f2max_pm2 = (double)f2m;
    vmax[0] = vm0; vmax[1] = vm1; vmax[2] = vm2;
  }
  out->dt_pm2 = dt_crit(0.5f, (float)out->f2max_pm2, a_mid);
  out->t_pm2 = omp_get_wtime() - t0;
  t0 = omp_get_wtime();
  // classification (kick.f90:108-138)
  std::vector<int> ires;
  classify(G, rhoc, ires, out->napm);
  const int64_t ns3 = (int64_t)ires.size();
  const int64_t ns_run = boxes_frac > 0 ? std::max<int64_t>(1, (int64_t)(ns3 * boxes_frac)) : ns3;
  if (G.pm3_on && (only & 4)) {
    std::vector<std::vector<float>> g3(8);
    for (int c = 2; c <= 5; ++c)
      if (out->napm[c] > 0) {
        g3[c].resize(G.nft[c] * G.nft[c] * (G.nft[c] / 2 + 1));
        green_3d(g3[c].data(), G.nft[c], G.apm3f, G.apm2 * (float)RSF[c], 1.f / (float)RSF[c]);
      }
    T f2m = 0, vm0 = 0, vm1 = 0, vm2 = 0;
    int64_t e = 0, mfx = 0;
    double md = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : f2m, vm0, vm1, vm2) reduction(| : e) reduction(+ : mfx, md)
    for (int64_t s = 0; s < ns_run; ++s) {
      BoxWork<T> w;
      Box b = make_pm3_box(G, s, ires[s]);
      box_density<T, XT>(G, C, xp, b, w, fixed, e, mfx, md);
      if (dbg_level == 3 && dbg_box == s && dbg_what == 0) dump(w.dens);
      T f2t = 0;
      box_force<T>(b, g3[ires[s]].data(), w, f2t);
      if (dbg_level == 3 && dbg_box == s && dbg_what == 1) dump(w.dens);
      if (dbg_level == 3 && dbg_box == s && dbg_what == 2) dump(w.force);
      T vm[3] = {0, 0, 0};
      box_interp<T, XT>(G, C, xp, vp, b, w, a_mid, dt, vm, e);
      f2m = std::max(f2m, f2t);
      vm0 = std::max(vm0, vm[0]);
      vm1 = std::max(vm1, vm[1]);
      vm2 = std::max(vm2, vm[2]);
    }
    err |= e;
    out->mass[2] = fixed ? std::ldexp((double)mfx, -FIXED_SHIFT) : md;
    out->f2max_pm3 = (double)f2m;
    vmax[0] = vm0; vmax[1] = vm1; vmax[2] = vm2;
  }
  out->dt_pm3 = dt_crit(0.5f, (float)out->f2max_pm3, a_mid);
  out->t_pm3 = omp_get_wtime() - t0;
  t0 = omp_get_wtime();
  if (G.pp_on && (only & 8)) {
    T f2m = 0, vm0 = 0, vm1 = 0, vm2 = 0;
    int64_t e = 0, npairs = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : f2m, vm0, vm1, vm2) reduction(| : e) reduction(+ : npairs)
    for (int64_t s = 0; s < ns_run; ++s) {
      Box b = make_pm3_box(G, s, ires[s]);
      T f2t = 0, vm[3] = {0, 0, 0};
      pp_box<T, XT>(G, C, xp, vp, b, a_mid, dt, f2t, vm, npairs, e);
      f2m = std::max(f2m, f2t);
      vm0 = std::max(vm0, vm[0]);
      vm1 = std::max(vm1, vm[1]);
      vm2 = std::max(vm2, vm[2]);
    }
    err |= e;
    out->f2max_pp = (double)f2m;
    out->pp_pairs = npairs;
    vmax[0] = vm0; vmax[1] = vm1; vmax[2] = vm2;
  }
  out->dt_pp = dt_crit(0.05f, (float)out->f2max_pp, a_mid);
  out->t_pp = omp_get_wtime() - t0;
  for (int d = 0; d < 3; ++d) out->vmax[d] = (double)vmax[d];
  const float vm = (float)std::max({vmax[0], vmax[1], vmax[2]});
  out->dt_vmax = 0.9f * 14 / vm;  // kick.f90:314
  out->vz_max = (float)vmax[2];
  out->err = err;
  return err ? CUBE_E_RANGE : 0;
}

}  // namespace oracle

extern "C" {

// kick.f90 in FP32 (the reference's kinds).  deposit_fixed selects the int64
// fixed-point deposit that the chosen GPU form uses.
int oracle_kick(const cube_params* p, const void* xp, float* vp, const int32_t* rhoc, float dt, float a_mid,
                int deposit_fixed, int only, double boxes_frac, oracle_kick_out* out, int dbg_level, int64_t dbg_box,
                int dbg_what, float* dbg_out, int64_t dbg_n) {
  Geo G = make_geo(p);
  if (G.izipx == 1)
    return kick_impl<float, int8_t>(G, (const int8_t*)xp, vp, rhoc, dt, a_mid, deposit_fixed != 0, only, boxes_frac,
                                    out, dbg_level, dbg_box, dbg_what, dbg_out, dbg_n);
  return kick_impl<float, int16_t>(G, (const int16_t*)xp, vp, rhoc, dt, a_mid, deposit_fixed != 0, only, boxes_frac, out,
                                   dbg_level, dbg_box, dbg_what, dbg_out, dbg_n);
}

// kick.f90 in FP64 throughout (the FP64 oracle).
int oracle_kick64(const cube_params* p, const void* xp, double* vp, const int32_t* rhoc, float dt, float a_mid, int only,
                  oracle_kick_out* out, int dbg_level, int64_t dbg_box, int dbg_what, float* dbg_out, int64_t dbg_n) {
  Geo G = make_geo(p);
  if (G.izipx == 1)
    return kick_impl<double, int8_t>(G, (const int8_t*)xp, vp, rhoc, dt, a_mid, false, only, 0.0, out, dbg_level,
                                     dbg_box, dbg_what, dbg_out, dbg_n);
  return kick_impl<double, int16_t>(G, (const int16_t*)xp, vp, rhoc, dt, a_mid, false, only, 0.0, out, dbg_level,
                                    dbg_box, dbg_what, dbg_out, dbg_n);
}

// ZIPV codec (utilities/pp_subtile.f90:61,125), FP64 as the reference, nvbin=2^16.
int oracle_zipv_encode(const float* v, int16_t* code, int64_t n, float sigma_vi) {
  const double sc = std::sqrt(M_PI / 2) / ((double)sigma_vi * 2.5);
  for (int64_t i = 0; i < n; ++i) code[i] = (int16_t)std::llround((double)65535.f * std::atan(sc * (double)v[i]) / M_PI);
  return 0;
}
int oracle_zipv_decode(const int16_t* code, float* v, int64_t n, float sigma_vi) {
  const double sc = std::sqrt(M_PI / 2) / ((double)sigma_vi * 2.5);
  for (int64_t i = 0; i < n; ++i) v[i] = (float)(std::tan(M_PI * (double)(float)code[i] / (double)65535.f) / sc);
  return 0;
}

// Subtile classes (kick.f90:108-133).
int oracle_classify(const cube_params* p, const int32_t* rhoc, int32_t* ires_out, int32_t* napm) {
  Geo G = make_geo(p);
  std::vector<int> ires;
  classify(G, rhoc, ires, napm);
  for (size_t i = 0; i < ires.size(); ++i) ires_out[i] = ires[i];
  return 0;
}

}  // extern "C"
