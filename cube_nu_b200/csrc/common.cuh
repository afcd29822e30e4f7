// Device-side geometry and helpers shared by the CUBE step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cube_gpu.h"

namespace cube {

// ratio_sf, parameters.f90:26 (1-based; class iapm uses RSF[iapm]).
__host__ __device__ inline int rsf_of(int iapm) {
  // {0, 1, 2, 4, 6, 8, 12, 16}[iapm & 7], without a local-memory table
  const int i = iapm & 7;
  return i <= 2 ? i : i == 3 ? 4 : i == 4 ? 6 : i == 5 ? 8 : i == 6 ? 12 : 16;
}

// Geometry derived from cube_params (parameters.f90:57-82).  Plain struct passed to
// kernels by value.
struct Geo {
  int ng, rcs, nnt, nns, ncb, ngb, nc, nt, ntt, ngp, ngt;
  int izipx;
  int nfp[8], nfb[8], nft[8];
  float app, apm1c, apm2, apm3f, mass_p, f_nu;
  double x_res;      // 2^(-8 izipx) coarse cells per code unit
  double inv_step;   // 1/(x_res*ratio_cs): code units per fine cell
  uint32_t zmask;    // 0xff or 0xffff
  int64_t ncells;    // nc^3
  // The part of the box this context steps (cube_params.nslab/slab): tiles [tile0, tile1),
  // their cells [c0, c1) in storage order and subtiles [s0, s1).  The whole box with one
  // slab; other cells hold ghost copies (or nothing).
  int nslab, tile0, tile1, s0, s1;
  int64_t c0, c1;
};

// Whether storage cell c belongs to this context's slab.
__host__ __device__ inline bool owned_cell(const Geo& G, int64_t c) { return c >= G.c0 && c < G.c1; }

// Cell `slot` of a ghost-exchange layer: the ncb cell layers lz0 .. lz0+ncb-1 of every tile
// of tile layer tz, in storage order.  Within a tile the cells of consecutive lz are
// consecutive in storage, so the layer is nnt^2 runs of ncb*nt^2 cells.
__host__ __device__ inline int64_t layer_cell(const Geo& G, int tz, int lz0, int64_t slot) {
  const int64_t run = (int64_t)G.ncb * G.nt * G.nt;
  const int64_t t = slot / run;
  const int64_t T = (int64_t)tz * G.nnt * G.nnt + t;
  return T * G.nt * G.nt * G.nt + (int64_t)lz0 * G.nt * G.nt + (slot - t * run);
}

// Per-step scalars, written by the host into device memory at the start of every step
// (one small copy, which a captured step graph replays), so that no kernel of the step
// takes them by value.  The host derives dt_mid, nlayer and the PP factors exactly as the
// reference does (drift.f90:21,26; kick.f90:283-285).
struct StepDev {
  float dt, dt_old, a_mid, vz_max;
  float dt_mid;       // (dt_old + dt) / 2
  int nlayer;         // 2*ceiling(dt_mid*vz_max/ratio_cs)+2
  float pp_mass;      // PP force factor (mass_p, times (1-f_nu)^2 with neutrinos)
  float pp_vscale;    // a_mid*dt/6/pi
};

__host__ __device__ inline int wrapi(int a, int n) {
  a %= n;
  return a < 0 ? a + n : a;
}

// Storage index of global coarse cell (gx,gy,gz) in the reference order
// rhoc(nt,nt,nt,nnt,nnt,nnt): tile z,y,x outer, then cell z,y,x (x fastest).
__host__ __device__ inline int64_t cell_index(const Geo& G, int gx, int gy, int gz) {
  gx = wrapi(gx, G.nc);
  gy = wrapi(gy, G.nc);
  gz = wrapi(gz, G.nc);
  const int tx = gx / G.nt, ty = gy / G.nt, tz = gz / G.nt;
  const int lx = gx - tx * G.nt, ly = gy - ty * G.nt, lz = gz - tz * G.nt;
  return ((((int64_t)(tz * G.nnt + ty) * G.nnt + tx) * G.nt + lz) * G.nt + ly) * G.nt + lx;
}

// Inverse of cell_index: global coarse cell coordinates (0-based).  In 32-bit unsigned
// arithmetic: contexts hold fewer than 2^32 coarse cells (checked at creation).
__host__ __device__ inline void cell_coords(const Geo& G, int64_t c, int& gx, int& gy, int& gz) {
  const unsigned nt = (unsigned)G.nt, nt2 = nt * nt, nnt = (unsigned)G.nnt;
  const unsigned cc = (unsigned)c;
  const unsigned t = cc / (nt2 * nt), r = cc - t * (nt2 * nt);
  const unsigned lz = r / nt2, r2 = r - lz * nt2, ly = r2 / nt, lx = r2 - ly * nt;
  const unsigned t1 = t / nnt, tx = t - t1 * nnt, tz = t1 / nnt, ty = t1 - tz * nnt;
  gx = (int)(tx * nt + lx);
  gy = (int)(ty * nt + ly);
  gz = (int)(tz * nt + lz);
}

// Storage index of the neighbour (dx, dy, dz) of storage cell c, whose tile-local
// coordinates are l: an offset within the tile, cell_index across a tile face.
__host__ __device__ inline int64_t nbr_cell(const Geo& G, int64_t c, const int l[3], const int g[3], int dx, int dy,
                                            int dz) {
  if ((unsigned)(l[0] + dx) < (unsigned)G.nt && (unsigned)(l[1] + dy) < (unsigned)G.nt &&
      (unsigned)(l[2] + dz) < (unsigned)G.nt)
    return c + ((int64_t)dz * G.nt + dy) * G.nt + dx;
  return cell_index(G, g[0] + dx, g[1] + dy, g[2] + dz);
}

// ZIPX decode, kick.f90:627-628: (int(xp+ishift,izipx)+rshift)*x_resolution equals
// ((unsigned)xp + 0.5) * 2^(-8 izipx), an exact double.
__device__ __forceinline__ double zfrac(int code, const Geo& G) {
  return ((double)((uint32_t)code & G.zmask) + 0.5) * G.x_res;
}

__device__ __forceinline__ int load_code(const void* xp, int izipx, int64_t i) {
  return izipx == 1 ? (int)((const int8_t*)xp)[i] : (int)((const int16_t*)xp)[i];
}

__device__ __forceinline__ void store_code(void* xp, int izipx, int64_t i, int v) {
  if (izipx == 1) ((int8_t*)xp)[i] = (int8_t)v;
  else ((int16_t*)xp)[i] = (int16_t)v;
}

// TSC weights with the reference's FP32 arithmetic (particle_mesh.f90:56-62):
// dx1=(1-l)^2/2, dx3=l^2/2, dx2=1-dx1-dx3 with l=xpos-floor(xpos).
__device__ __forceinline__ int tsc_weights(double xpos, float w[3]) {
  const double fl = floor(xpos);
  const float l = (float)(xpos - fl);
  const float a = __fsub_rn(1.f, l);
  w[0] = __fmul_rn(__fmul_rn(a, a), 0.5f);
  w[2] = __fmul_rn(__fmul_rn(l, l), 0.5f);
  w[1] = __fsub_rn(__fsub_rn(1.f, w[0]), w[2]);
  return (int)fl + 1;  // idx(:,2), 1-based
}

// vp + dv*a_mid*dt/6/pi with the last division by real(8) pi (kick.f90:797).
__device__ __forceinline__ float kick_add(float v, float dv, float a_mid, float dt) {
  const float t = __fdiv_rn(__fmul_rn(__fmul_rn(dv, a_mid), dt), 6.f);
  return (float)__dadd_rn((double)v, __ddiv_rn((double)t, 3.141592653589793));
}

// Fixed-point weight round(w * 2^40) (round half to even, as the oracle's llrint), for
// 0 <= w <= 2^23: the scaling by 2^40 is exact in FP32 and one conversion rounds.
__device__ __forceinline__ unsigned long long fixed40(float w) {
  return (unsigned long long)__float2ll_rn(__fmul_rn(w, 1099511627776.f));
}

// Non-negative float max through integer atomics.
__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

__device__ __forceinline__ void set_err(unsigned* err, unsigned bit) { atomicOr(err, bit); }

// Gradient weights (parameters.f90:53-54), real4.
#define CUBE_W_ALPHA (4.f / 3.f)

}  // namespace cube
