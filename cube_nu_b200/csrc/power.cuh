// Power spectrum of the device-resident particles for one image (nn=1):
//   utilities/cicpower.f90:76-98    CIC density on an nw^3 periodic mesh, with the
//                                   reference's real(4) position arithmetic
//   utilities/cicpower.f90:165-181  delta = rho / mean - 1, mean summed in real(8)
//   utilities/powerspectrum.f90:140-190  auto_power binning: nint(|k|) bins, the
//                                   half-spectrum duplicates skipped, shot noise with
//                                   the mass-assignment window C1k
//   utilities/powerspectrum.f90:212-259  pk_correction alias integral over the
//                                   (i >= j >= k) wedge with n_int images per side
// Per-mode arithmetic follows the reference's kinds; the bin sums accumulate in double
// (the reference sums in real(4)), so they are at least as accurate.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace cube {

// CIC deposit.  FIXED: int64 fixed point round(w*2^40) into a dense nw^3 array (order
// independent); else FP32 atomics into the pitched real mesh (row pitch pr, plane pl).
template <bool FIXED>
__global__ void k_cic_deposit(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                              void* __restrict__ rho, int nw, int pr, int64_t pl) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  const float fnw = (float)nw, fnc = (float)G.nc;
  int i1[3];
  float d1[3], d2[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // integer cell + real(8) ZIPX decode, assigned to real(4) (cicpower.f90:79-80)
    float pos = __double2float_rn((double)g[d] + zfrac(load_code(xp, G.izipx, 3 * ip + d), G));
    pos = __fsub_rn(__fdiv_rn(__fmul_rn(pos, fnw), fnc), 0.5f);
    const float fl = floorf(pos);
    i1[d] = (int)fl;  // 0-based lower corner, in [-1, nw-1]
    d1[d] = __fsub_rn(fl + 1.f, pos);
    d2[d] = __fsub_rn(1.f, d1[d]);
  }
  const int x0 = wrapi(i1[0], nw), x1 = wrapi(i1[0] + 1, nw);
  const int y0 = wrapi(i1[1], nw), y1 = wrapi(i1[1] + 1, nw);
  const int z0 = wrapi(i1[2], nw), z1 = wrapi(i1[2] + 1, nw);
  const int xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        const float w = __fmul_rn(__fmul_rn(a ? d2[0] : d1[0], b ? d2[1] : d1[1]), c ? d2[2] : d1[2]);
        const int64_t idx = (int64_t)zs[c] * pl + (int64_t)ys[b] * pr + xs[a];
        if (FIXED) {
          const long long q = (long long)fixed40(w);  // round(w * 2^40)
          atomicAdd(reinterpret_cast<unsigned long long*>(rho) + idx, (unsigned long long)q);
        } else {
          atomicAdd(reinterpret_cast<float*>(rho) + idx, w);
        }
      }
}

// Deterministic block sum in double: fixed-order tree over the block's threads.
__device__ __forceinline__ double block_sum_det(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  return sh[0];
}

// Density in the float mesh (from the fixed-point sums when FIXED) and per-block
// double partial sums of it, in a fixed order.  blockDim = 256.
template <bool FIXED>
__global__ void k_pk_density(const long long* __restrict__ acc, float* __restrict__ mesh, int nw, int pr, int64_t pl,
                             double* __restrict__ partial) {
  __shared__ double sh[256];
  const int64_t n3 = (int64_t)nw * nw * nw;
  double s = 0.0;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n3; q += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % nw);
    const int64_t yz = q / nw;
    const int y = (int)(yz % nw), z = (int)(yz / nw);
    float* m = mesh + (int64_t)z * pl + (int64_t)y * pr + x;
    float r;
    if (FIXED) {
      r = __double2float_rn((double)acc[q] * 0x1p-40);
      *m = r;
    } else {
      r = *m;
    }
    s += (double)r;
  }
  const double t = block_sum_det(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// Sum of the per-block partials by one block, in a fixed order.
__global__ void k_pk_sum_partials(const double* __restrict__ partial, int n, double* __restrict__ out) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  const double t = block_sum_det(s, sh);
  if (threadIdx.x == 0) *out = t;
}

// Order-preserving int image of a float (for atomicMin/atomicMax).
__device__ __forceinline__ int float_order_key(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}

// delta = rho/mean - 1 in place (cicpower.f90:180: real(4)/real(8) - 1 -> real(4)),
// with min/max keys in mm[0], mm[1].
__global__ void k_pk_delta(float* __restrict__ mesh, int nw, int pr, int64_t pl, double mean, int* __restrict__ mm) {
  const int64_t n3 = (int64_t)nw * nw * nw;
  float lo = 3.0e38f, hi = -3.0e38f;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n3; q += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(q % nw);
    const int64_t yz = q / nw;
    const int y = (int)(yz % nw), z = (int)(yz / nw);
    float* m = mesh + (int64_t)z * pl + (int64_t)y * pr + x;
    const float d = __double2float_rn(__dsub_rn(__ddiv_rn((double)*m, mean), 1.0));
    *m = d;
    lo = fminf(lo, d);
    hi = fmaxf(hi, d);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, float_order_key(lo));
    atomicMax(mm + 1, float_order_key(hi));
  }
}

// auto_power binning (powerspectrum.f90:154-187) over the half spectrum c(kz,ky,kx)
// (row pitch pc, plane pitch plc, complex).  Per bin: count, sum kr, sum |d_k|^2,
// sum (|d_k|^2 - Dk), accumulated in double; bins[4*(nbin+1)] must start at zero.
// Dynamic shared memory: 4*(nbin+1) doubles.
__global__ void k_pk_bin(const float2* __restrict__ c, int nw, int pc, int64_t plc, int nbin, float np_f,
                         int n_interp, double* __restrict__ bins) {
  extern __shared__ double sb[];
  const int nb4 = 4 * (nbin + 1);
  for (int i = threadIdx.x; i < nb4; i += blockDim.x) sb[i] = 0.0;
  __syncthreads();
  const int nh = nw / 2 + 1, nyq = nw / 2;
  const float fn = (float)nw;
  const double PI = 3.141592653589793;
  const int64_t nm = (int64_t)nw * nw * nh;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(m % nh);
    const int64_t jk = m / nh;
    const int j = (int)(jk % nw), k = (int)(jk / nw);
    if (i == 0 && j == 0 && k == 0) continue;  // zero frequency
    if ((i == 0 || i == nyq) && j > nyq) continue;
    if ((i == 0 || i == nyq) && (j == 0 || j == nyq) && k > nyq) continue;
    const int mm[3] = {i, j, k};
    float kx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) kx[d] = (float)((mm[d] + nyq) % nw - nyq);
    const float kr = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(kx[0], kx[0]), __fmul_rn(kx[1], kx[1])),
                                          __fmul_rn(kx[2], kx[2])));
    const int ib = (int)lroundf(kr);
    const float2 v = c[(int64_t)k * plc + (int64_t)j * pc + i];
    const float re = __fdiv_rn(__fdiv_rn(__fdiv_rn(v.x, fn), fn), fn);
    const float im = __fdiv_rn(__fdiv_rn(__fdiv_rn(v.y, fn), fn), fn);
    const float amp = __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im));
    float c1k[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double s = sin(PI * (double)kx[d] / (double)nw);
      const double s2 = s * s;
      if (n_interp == 1) c1k[d] = 1.f;
      else if (n_interp == 2) c1k[d] = __double2float_rn(1.0 - (double)(2.f / 3.f) * s2);
      else c1k[d] = __double2float_rn(1.0 - s2 + (double)(2.f / 15.f) * (s2 * s2));
    }
    const float dk = __fdiv_rn(__fmul_rn(__fmul_rn(c1k[0], c1k[1]), c1k[2]), np_f);
    double* b = sb + 4 * ib;
    atomicAdd(b + 0, 1.0);
    atomicAdd(b + 1, (double)kr);
    atomicAdd(b + 2, (double)amp);
    atomicAdd(b + 3, (double)__fsub_rn(amp, dk));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb4; i += blockDim.x)
    if (sb[i & ~3] != 0.0) atomicAdd(bins + i, sb[i]);
}

// gcc's integer power by squaring (gfortran real**integer).
__device__ __forceinline__ float powi_f(float x, int n) {
  float y = (n & 1) ? x : 1.f;
  while (n >>= 1) {
    x = __fmul_rn(x, x);
    if (n & 1) y = __fmul_rn(y, x);
  }
  return y;
}

constexpr int PK_MAX_NINT = 4;

// pk_correction's integral (powerspectrum.f90:228-252): one block per (i, j) with
// j <= i <= nyq, threads over k <= j.  Per bin: count, sum kmag, sum Wk2Pk/Pk, in
// double; cb[3*(nbin+1)] must start at zero.  Dynamic shared memory: 3*(nbin+1) doubles.
template <int NI>
__global__ void k_pk_alias(int nw, int nbin, float alpha, int p2, double* __restrict__ cb) {
  constexpr int n_int = NI, ni = 2 * NI + 1;
  extern __shared__ double sc[];
  const int64_t pidx = blockIdx.x;
  int i = (int)((sqrt(8.0 * (double)pidx + 1.0) - 1.0) * 0.5);
  while ((int64_t)(i + 1) * (i + 2) / 2 <= pidx) ++i;
  while ((int64_t)i * (i + 1) / 2 > pidx) --i;
  const int j = (int)(pidx - (int64_t)i * (i + 1) / 2);
  const float fi = (float)i, fj = (float)j;
  const float ij2 = __fadd_rn(__fmul_rn(fi, fi), __fmul_rn(fj, fj));
  const int blo = (int)lroundf(__fsqrt_rn(__fadd_rn(ij2, 0.f)));
  const int bhi = (int)lroundf(__fsqrt_rn(__fadd_rn(ij2, __fmul_rn(fj, fj))));
  for (int b = blo * 3 + threadIdx.x; b < (bhi + 1) * 3; b += blockDim.x) sc[b] = 0.0;
  __syncthreads();
  const double PI = 3.141592653589793;
  // sinc and squares of the alias images along x (i) and y (j) are the same for every k
  float sx[ni], sy[ni], qx[ni], qy[ni];
#pragma unroll
  for (int n = 0; n < ni; ++n) {
    const float ax = __fadd_rn(fi, (float)((n - n_int) * nw)), ay = __fadd_rn(fj, (float)((n - n_int) * nw));
    const float kx = __double2float_rn(PI * (double)ax / (double)nw), ky = __double2float_rn(PI * (double)ay / (double)nw);
    sx[n] = kx == 0.f ? 1.f : __fdiv_rn(sinf(kx), kx);
    sy[n] = ky == 0.f ? 1.f : __fdiv_rn(sinf(ky), ky);
    qx[n] = __fmul_rn(ax, ax);
    qy[n] = __fmul_rn(ay, ay);
  }
  for (int k = threadIdx.x; k <= j; k += blockDim.x) {
    const float fk = (float)k;
    const float kmag = __fsqrt_rn(__fadd_rn(ij2, __fmul_rn(fk, fk)));
    const int ib = (int)lroundf(kmag);
    const float pk = powf(kmag, alpha);
    float sz[ni], qz[ni];
#pragma unroll
    for (int n = 0; n < ni; ++n) {
      const float az = __fadd_rn(fk, (float)((n - n_int) * nw));
      const float kz = __double2float_rn(PI * (double)az / (double)nw);
      sz[n] = kz == 0.f ? 1.f : __fdiv_rn(sinf(kz), kz);
      qz[n] = __fmul_rn(az, az);
    }
    float w2p = 0.f;
#pragma unroll
    for (int a = 0; a < ni; ++a)
#pragma unroll
      for (int b = 0; b < ni; ++b) {
        const float pab = __fmul_rn(sx[a], sy[b]);
        const float qab = __fadd_rn(qx[a], qy[b]);
#pragma unroll
        for (int cz = 0; cz < ni; ++cz) {
          const float kmagn = __fsqrt_rn(__fadd_rn(qab, qz[cz]));
          const float w = powi_f(__fmul_rn(pab, sz[cz]), p2);
          w2p = __fadd_rn(w2p, __fmul_rn(w, powf(kmagn, alpha)));
        }
      }
    double* s = sc + 3 * ib;
    atomicAdd(s + 0, 1.0);
    atomicAdd(s + 1, (double)kmag);
    atomicAdd(s + 2, (double)__fdiv_rn(w2p, pk));
  }
  __syncthreads();
  for (int b = blo * 3 + threadIdx.x; b < (bhi + 1) * 3; b += blockDim.x)
    if (sc[b - b % 3] != 0.0) atomicAdd(cb + b, sc[b]);
}

}  // namespace cube
