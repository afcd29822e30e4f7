// Zel'dovich initial conditions on the device (utilities/ic.f90), one image.
//
//   noise U[0,1) per IC cell from Philox4x32-10 (Salmon et al. 2011), key = seed,
//     counter = pair index -> Box-Muller pairs along x (ic.f90:289-299)
//   multiplier sqrt(P(k)(nw/box)^3) * (-4 pi / k_d^2) (ic.f90:363-437), applied by the
//     same staged FFT Poisson solve as the PM levels (normalised by nw three times as
//     pencil_fft_backward does)
//   particles on the lattice: corner gradient of phi (ic.f90:665-667), displacement
//     -grad/(8 nic pi ratio_cs) coarse cells, velocity -grad/(8 pi nic)*vfactor, ZIPX code
//     floor(xq/x_resolution), PID (ic.f90:700-729), arrival key (ilayer,k,j,i) in the
//     destination tile's lattice frame; the drift's sort kernels then place them in the
//     reference order.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace cube {

// Philox4x32-10 block cipher (public algorithm, Random123).
__host__ __device__ inline uint4 philox4x32_10(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)M0 * c.x, p1 = (uint64_t)M1 * c.z;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

// uniform [0,1) with 24 bits
__host__ __device__ inline float u24(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

// Noise and Box-Muller into the real IC mesh (row pitch pr, plane pitch pl floats); pairs
// (2m, 2m+1) along x.  One thread per pair.
__global__ void k_ic_noise(float* __restrict__ mesh, int nw, int pr, int64_t pl, uint2 key) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t npair = (int64_t)nw * nw * nw / 2;
  if (m >= npair) return;
  const uint4 r = philox4x32_10(make_uint4((uint32_t)m, (uint32_t)(m >> 32), 0u, 0u), key);
  const float u1 = u24(r.x), u2 = u24(r.y);
  const double th = 2.0 * 3.141592653589793 * (double)u1;
  const double rr = sqrt(-2.0 * log(1.0 - (double)u2));
  const int64_t i = 2 * m;
  const int x = (int)(i % nw), y = (int)((i / nw) % nw), z = (int)(i / ((int64_t)nw * nw));
  float* row = mesh + (int64_t)z * pl + (int64_t)y * pr;
  row[x] = (float)(rr * cos(th));
  row[x + 1] = (float)(rr * sin(th));
}

// Multiplier table g[kz][ky][kx] (dense, nw/2+1 fastest): sqrt(P(kr)(nw/box)^3)*(-4pi/kd^2),
// P interpolated linearly in log-log from (lk, lp) (ic.f90 interp_tf), zero at k=0.
__global__ void k_ic_multiplier(float* __restrict__ g, int nw, float box, const double* __restrict__ lk,
                                const double* __restrict__ lp, int npk) {
  const int nh = nw / 2 + 1;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nw * nw * nh) return;
  const int kx = (int)(i % nh), ky0 = (int)((i / nh) % nw), kz0 = (int)(i / ((int64_t)nh * nw));
  const int ky = (ky0 + nw / 2) % nw - nw / 2, kz = (kz0 + nw / 2) % nw - nw / 2;  // ic.f90:372-374
  if (kx == 0 && ky == 0 && kz == 0) {
    g[i] = 0.f;
    return;
  }
  const double PI = 3.141592653589793;
  const double kr = 2.0 * PI * sqrt((double)kx * kx + (double)ky * ky + (double)kz * kz) / (double)box;
  const double lkr = log(kr);
  int a = 0, b = npk - 1;
  while (b - a > 1) {
    const int c = (a + b) / 2;
    if (lkr > lk[c]) a = c;
    else b = c;
  }
  const double lpv = lp[a] + (lp[b] - lp[a]) * (lkr - lk[a]) / (lk[b] - lk[a]);
  const double tf = sqrt(exp(lpv) * pow((double)nw / (double)box, 3.0));
  const double sx = 2 * sin(PI * kx / nw), sy = 2 * sin(PI * ky / nw), sz = 2 * sin(PI * kz / nw);
  const double kd = fmax(sx * sx + sy * sy + sz * sz, 1.0 / ((double)nw * nw));
  g[i] = (float)(tf * (-4.0 * PI / kd));
}

struct ICArgs {
  int nw, nlat, step, np_nc, nic, nlayer;
  float vf;
  double lat_off;  // (0.5/nic)/ratio_cs
};

// Corner gradient at lattice point L (ic.f90:665-667): 0.5*sum over the 2x2x2 block.
__device__ __forceinline__ void ic_grad(const float* phi, int nw, int pf, int64_t pl, int step, int Lx, int Ly, int Lz,
                                        float g[3]) {
  const int ix[2] = {wrapi(step * Lx - 1, nw), wrapi(step * Lx, nw)};
  const int iy[2] = {wrapi(step * Ly - 1, nw), wrapi(step * Ly, nw)};
  const int iz[2] = {wrapi(step * Lz - 1, nw), wrapi(step * Lz, nw)};
  float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const float v = phi[(int64_t)iz[c] * pl + (int64_t)iy[b] * pf + ix[a]];
        gx += (a ? 0.5f : -0.5f) * v;
        gy += (b ? 0.5f : -0.5f) * v;
        gz += (c ? 0.5f : -0.5f) * v;
      }
  g[0] = gx;
  g[1] = gy;
  g[2] = gz;
}

// max |gradphi| per axis (for vz_max and the thread-safe layer count, ic.f90:575-590)
__global__ void k_ic_gradmax(const float* __restrict__ phi, int pf, int64_t pl, ICArgs A, float* __restrict__ gmax) {
  const int64_t L = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n3 = (int64_t)A.nlat * A.nlat * A.nlat;
  float g[3] = {0.f, 0.f, 0.f};
  if (L < n3) {
    const int Lx = (int)(L % A.nlat), Ly = (int)((L / A.nlat) % A.nlat), Lz = (int)(L / ((int64_t)A.nlat * A.nlat));
    ic_grad(phi, A.nw, pf, pl, A.step, Lx, Ly, Lz, g);
  }
  for (int d = 0; d < 3; ++d) {
    float v = fabsf(g[d]);
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomic_max_pos(gmax + d, v);
  }
}

// One particle per lattice point: code, velocity, PID, destination cell, arrival key and
// count.  Writes the unsorted source arrays; the drift's scatter/sort/gather place them.
__global__ void k_ic_particles(Geo G, const float* __restrict__ phi, int pf, int64_t pl, ICArgs A, void* __restrict__ xp,
                               float* __restrict__ vp, int64_t* __restrict__ pid, int32_t* __restrict__ dest,
                               uint64_t* __restrict__ key, int32_t* __restrict__ count, unsigned* err) {
  const int64_t L = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n3 = (int64_t)A.nlat * A.nlat * A.nlat;
  if (L >= n3) return;
  const int Lc[3] = {(int)(L % A.nlat), (int)((L / A.nlat) % A.nlat), (int)(L / ((int64_t)A.nlat * A.nlat))};
  float g[3];
  ic_grad(phi, A.nw, pf, pl, A.step, Lc[0], Lc[1], Lc[2], g);
  const double PI = 3.141592653589793;
  int cell[3];
  int64_t iq[3];
  uint64_t kk[3];
  const int npt = G.nt * A.np_nc, npb = A.np_nc;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // xq = L/np_nc + (0.5/nic)/ratio_cs - gradphi/(8 nic pi ratio_cs), coarse units (ic.f90:700)
    const double xq = (double)Lc[d] / A.np_nc + A.lat_off - (double)g[d] / (8.0 * A.nic * PI * G.rcs);
    const double fl = floor(xq);
    cell[d] = wrapi((int)fl, G.nc);
    const long long code = (long long)floor(xq / G.x_res);  // floor(xq/x_resolution), kind=8 then wrap
    store_code(xp, G.izipx, 3 * L + d, (int)(code & (long long)G.zmask));
    vp[3 * L + d] = (float)((-(double)g[d] / (8.0 * PI * A.nic)) * (double)A.vf);  // ic.f90:722
    iq[d] = ((int64_t)(G.rcs / A.np_nc) * Lc[d]) % G.ng;
    // lattice coordinate in the destination tile's frame: the copy within a lattice span
    const int tile = cell[d] / G.nt;
    int lloc = Lc[d] - tile * npt;
    const double xloc = (double)cell[d] - (double)tile * G.nt + (xq - fl);
    const double lpos = (lloc + 0.5) / A.np_nc;
    if (lpos - xloc > 0.5 * G.nc) lloc -= A.nlat;
    else if (xloc - lpos > 0.5 * G.nc) lloc += A.nlat;
    if (lloc < -npb || lloc >= npt + npb) set_err(err, CUBE_DEVERR_DRIFT_RANGE);
    kk[d] = (uint64_t)(lloc + npb);
  }
  pid[L] = iq[0] + (int64_t)G.ng * iq[1] + (int64_t)G.ng * G.ng * iq[2] + 1;
  const int64_t dc = cell_index(G, cell[0], cell[1], cell[2]);
  dest[L] = (int32_t)dc;
  key[L] = ((kk[2] % (uint64_t)A.nlayer) << 48) | (kk[2] << 32) | (kk[1] << 16) | kk[0];
  atomicAdd(&count[dc], 1);
}

}  // namespace cube
