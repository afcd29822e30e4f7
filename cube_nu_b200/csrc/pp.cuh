// PP short-range force (kick.f90:376-588) as a work queue over coarse cells, for the
// chosen form of the step.  Included by cube_gpu.cu after kernels.cuh.
//
// The pairs and the force law are those of k_pp: every physical particle sums the
// 0 < r^2 < range^2 pairs over the coarse cells its range reaches (range = 3.5/rsf fine
// cells of its subtile's class), cells in the order dz, dy, dx and particles in storage
// order within a cell.  The work is split by the occupancy of the particle's own cell:
//   * light cells (at most T particles): one thread per particle (k_ppq_light);
//   * heavy cells: their particles counting-sorted by the set of neighbour cells they reach
//     (k_ppq_sort_codes), then cut into items of B particles of one cell, pulled from a
//     device queue by a persistent kernel (k_ppq_heavy) whose block stages the candidate
//     cells' particles in shared memory in chunks of J and tests its B particles against
//     each chunk.  The queue is ordered by occupancy, largest first (log2 buckets), so the
//     long items start first and the tail is short.
// Both paths read the candidates' in-cell offsets, decoded once per step into a float4
// array (k_ppq_prep), test candidates four at a time as independent chains, defer the
// pairs in range to a per-thread shared-memory column and add them in candidate order,
// so each particle's pairs are summed with the same operations in the same order and the
// force does not depend on (T, B, J): the autotuner (cube_gpu.cu, pp_tune) picks the
// fastest shape per occupancy class freely.
#pragma once
#include "kernels.cuh"

namespace cube {

// In-cell offset of every particle in fine cells: (u + 0.5) * x_res * ratio_cs per
// coordinate, exact in FP32 for izipx <= 2 (at most 17 significant bits).
__global__ void k_ppq_prep(Geo G, int64_t np, const void* __restrict__ xp, float4* __restrict__ pfin) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  float f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) f[d] = __fmul_rn((float)zfrac(load_code(xp, G.izipx, 3 * ip + d), G), (float)G.rcs);
  pfin[ip] = make_float4(f[0], f[1], f[2], 0.f);
}

// One particle's PP state: its tile-local position xf (fine cells), the candidate cell
// range per dimension, its range and the accumulated force.  The candidate coordinate is
// (lq*ratio_cs) + offset with lq = l + d: exact in FP32 when lq + offset fits 24 bits (the
// FAST case of k_pp), so rv equals k_pp's FAST arithmetic bit for bit.
struct PPi {
  float xf[3];
  int l[3], lo[3], hi[3];
  float range, range2, coef_range, coef_app;  // range and F_ra_coef of range and app
  float acc[3];
  unsigned pairs, cand;  // of this particle (item): well below 2^32

  __device__ __forceinline__ void init(const Geo& G, const int g[3], const float4 fin, int iapm) {
    const float fi[3] = {fin.x, fin.y, fin.z};
    range = __fdiv_rn(3.5f, (float)rsf_of(iapm));  // apm3(iapm)
    range2 = __fmul_rn(range, range);
    coef_range = F_ra_coef(range);
    coef_app = F_ra_coef(G.app);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      l[d] = g[d] % G.nt;
      xf[d] = __fadd_rn((float)(l[d] * G.rcs), fi[d]);
      lo[d] = (fi[d] < range) ? -1 : 0;
      hi[d] = ((float)G.rcs - fi[d] < range) ? 1 : 0;
      acc[d] = 0.f;
    }
    pairs = cand = 0;
  }

  __device__ __forceinline__ bool needs(int dx, int dy, int dz) const {
    return dx >= lo[0] && dx <= hi[0] && dy >= lo[1] && dy <= hi[1] && dz >= lo[2] && dz <= hi[2];
  }

  // The force of one pair in range (separation rv, r2 = |rv|^2) added to acc.  Callers
  // that defer their pairs call it in candidate order, so the sums are k_pp's.
  __device__ __forceinline__ void accum(float rv0, float rv1, float rv2, float r2, float app) {
    const float rm = __fsqrt_rn(r2);
    const float sc = __fsub_rn(F_ra_c(rm, app, coef_app), F_ra_c(rm, range, coef_range));
    acc[0] = __fadd_rn(acc[0], __fmul_rn(__fdiv_rn(rv0, rm), sc));
    acc[1] = __fadd_rn(acc[1], __fmul_rn(__fdiv_rn(rv1, rm), sc));
    acc[2] = __fadd_rn(acc[2], __fmul_rn(__fdiv_rn(rv2, rm), sc));
  }

  // One candidate at in-cell offset p of the neighbour cell whose tile-local coarse
  // coordinates are (bx, by, bz) (= l + d), already multiplied by ratio_cs.
  __device__ __forceinline__ void pair(float bx, float by, float bz, const float4 p, float app) {
    const float rv0 = __fsub_rn(__fadd_rn(bx, p.x), xf[0]);
    const float rv1 = __fsub_rn(__fadd_rn(by, p.y), xf[1]);
    const float rv2 = __fsub_rn(__fadd_rn(bz, p.z), xf[2]);
    const float r2 = sumsq3(rv0, rv1, rv2);
    if (r2 > 0.f && r2 < range2) {
      accum(rv0, rv1, rv2, r2, app);
      ++pairs;
    }
  }

  // The candidates of every cell this particle's range reaches, in order (the sums of
  // k_pp), reading the decoded offsets; counts candidates.  c: the particle's storage cell.
  __device__ __forceinline__ void all_cells(const Geo& G, int64_t c, const int g[3], const int64_t* __restrict__ cstart,
                                            const float4* __restrict__ pfin) {
    for (int dz = lo[2]; dz <= hi[2]; ++dz)
      for (int dy = lo[1]; dy <= hi[1]; ++dy)
        for (int dx = lo[0]; dx <= hi[0]; ++dx) {
          const int64_t n = nbr_cell(G, c, l, g, dx, dy, dz);
          const int64_t s = cstart[n], e = cstart[n + 1];
          cand += (unsigned)(e - s);
          const float bx = (float)((l[0] + dx) * G.rcs), by = (float)((l[1] + dy) * G.rcs),
                      bz = (float)((l[2] + dz) * G.rcs);
          for (int64_t q = s; q < e; ++q) pair(bx, by, bz, pfin[q], G.app);
        }
  }
};

// The kick of one particle from its PP force (kick.f90:300-306); returns |F|^2 and |v|.
__device__ __forceinline__ float ppq_apply(const PPi& P, int64_t ip, const float* vin, float* vout, float mass_scale,
                                           float v_scale, float av[3]) {
  float f1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) f1[d] = __fmul_rn(P.acc[d], mass_scale);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float v = __fadd_rn(vin[3 * ip + d], __fmul_rn(f1[d], v_scale));
    vout[3 * ip + d] = v;
    av[d] = fabsf(v);
  }
  return sumsq3(f1[0], f1[1], f1[2]);
}

__device__ __forceinline__ int ppq_iapm(const Geo& G, const int g[3], const int32_t* ires) {
  int t[3], u[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    t[d] = g[d] / G.nt;
    u[d] = (g[d] - t[d] * G.nt) / G.ntt;
  }
  return ires[subtile_id(G, t, u)];
}

// Particles of light cells (count <= T), one thread each.  vin/vout: velocities before and
// after (the same array in a step; the tuner writes a scratch copy).  Pairs in range are
// deferred as in k_ppq_heavy: a thread keeps up to PPL_H of them (rv, r2) in its own
// shared-memory column and adds them with PPi::accum in candidate order when the column
// is full and at the end, so a warp runs the force of a pair once per PPL_H pairs of a
// lane rather than once per candidate that any of its lanes has in range.
constexpr int PPL_T = 128;  // threads per block
constexpr int PPL_H = 8;    // deferred pairs per thread
constexpr int PPL_U = 4;    // candidates evaluated together

__global__ void __launch_bounds__(PPL_T) k_ppq_light(Geo G, int64_t np, const int32_t* __restrict__ pcell,
                                                   const int64_t* __restrict__ cstart, const int32_t* __restrict__ ires,
                                                   const float4* __restrict__ pfin, const float* vin, float* vout,
                                                   const StepDev* __restrict__ sd, int heavy_t, float* f2max,
                                                   float* vmax, unsigned long long* npairs,
                                                   unsigned long long* ncand, const unsigned* __restrict__ abort) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool live = ip < np && !(abort && *abort);
  int c = 0;
  if (live) {
    c = pcell[ip];
    live = owned_cell(G, c) && cstart[c + 1] - cstart[c] <= heavy_t;
  }
  __shared__ float4 hb[PPL_H][PPL_T];
  float f2 = 0.f, av[3] = {0.f, 0.f, 0.f};
  PPi P;
  P.pairs = P.cand = 0;
  if (live) {
    int g[3];
    cell_coords(G, c, g[0], g[1], g[2]);
    P.init(G, g, pfin[ip], ppq_iapm(G, g, ires));
    int nh = 0;
    for (int dz = P.lo[2]; dz <= P.hi[2]; ++dz)
      for (int dy = P.lo[1]; dy <= P.hi[1]; ++dy)
        for (int dx = P.lo[0]; dx <= P.hi[0]; ++dx) {
          const int64_t n = nbr_cell(G, c, P.l, g, dx, dy, dz);
          const int64_t s = cstart[n], e = cstart[n + 1];
          P.cand += (unsigned)(e - s);
          const float bx = (float)((P.l[0] + dx) * G.rcs), by = (float)((P.l[1] + dy) * G.rcs),
                      bz = (float)((P.l[2] + dz) * G.rcs);
          for (int64_t q0 = s; q0 < e; q0 += PPL_U) {
            // PPL_U candidates as independent chains (loads in flight together, the tail
            // predicated off), their pairs then recorded in candidate order
            float rv[PPL_U][3], r2[PPL_U];
            bool hit[PPL_U];
#pragma unroll
            for (int u = 0; u < PPL_U; ++u) {
              const bool valid = q0 + u < e;
              const float4 p = pfin[valid ? q0 + u : q0];
              rv[u][0] = __fsub_rn(__fadd_rn(bx, p.x), P.xf[0]);
              rv[u][1] = __fsub_rn(__fadd_rn(by, p.y), P.xf[1]);
              rv[u][2] = __fsub_rn(__fadd_rn(bz, p.z), P.xf[2]);
              r2[u] = sumsq3(rv[u][0], rv[u][1], rv[u][2]);
              hit[u] = valid && r2[u] > 0.f && r2[u] < P.range2;
            }
#pragma unroll
            for (int u = 0; u < PPL_U; ++u)
              if (hit[u]) {
                if (nh == PPL_H) {
#pragma unroll 1
                  for (int h = 0; h < PPL_H; ++h) {
                    const float4 r = hb[h][threadIdx.x];
                    P.accum(r.x, r.y, r.z, r.w, G.app);
                  }
                  nh = 0;
                }
                hb[nh][threadIdx.x] = make_float4(rv[u][0], rv[u][1], rv[u][2], r2[u]);
                ++nh;
                ++P.pairs;
              }
          }
        }
#pragma unroll 1
    for (int h = 0; h < nh; ++h) {
      const float4 r = hb[h][threadIdx.x];
      P.accum(r.x, r.y, r.z, r.w, G.app);
    }
    f2 = ppq_apply(P, ip, vin, vout, sd->pp_mass, sd->pp_vscale, av);
  }
  block_max_to(f2, f2max);
  block_vmax(av, vmax);
  unsigned long long a = P.pairs, b = P.cand;  // warp sums in 64 bits
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0 && a) atomicAdd(npairs, a);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(ncand, b);
}

// ---- the heavy-cell queue ----
// Heavy cells (count > T) in descending log2(count) buckets.  q[0..31]: bucket counts,
// q[32..63]: bucket cursors, q[64]: heavy cells, q[65]: items (tiles of B particles),
// q[66]: the queue counter.
constexpr int PPQ_Q = 72;

// bucket of a count n >= 1: floor(log2 n), 0..31
__device__ __forceinline__ int ppq_bucket(int64_t n) { return 63 - __clzll((unsigned long long)n); }

// Cells [c0, c1): this rank's slab.
__global__ void k_ppq_bucket_count(const int64_t* __restrict__ cstart, int64_t c0, int64_t c1, int heavy_t,
                                   int* __restrict__ q) {
  const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  const int64_t n = cstart[c + 1] - cstart[c];
  if (n > heavy_t) atomicAdd(&q[ppq_bucket(n)], 1);
}

// One thread: cursors for descending buckets.
__global__ void k_ppq_bucket_scan(int* __restrict__ q) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int off = 0;
  for (int b = 31; b >= 0; --b) {
    q[32 + b] = off;
    off += q[b];
  }
  q[64] = off;
}

__global__ void k_ppq_bucket_fill(const int64_t* __restrict__ cstart, int64_t c0, int64_t c1, int heavy_t,
                                  int* __restrict__ q, int32_t* __restrict__ hlist) {
  const int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  const int64_t n = cstart[c + 1] - cstart[c];
  if (n > heavy_t) hlist[atomicAdd(&q[32 + ppq_bucket(n)], 1)] = (int32_t)c;
}

// Exclusive prefix of the items per heavy cell (ceil(count/B)), one block; hpre has
// nheavy+1 entries and q[65] receives the total.
__global__ void __launch_bounds__(1024) k_ppq_items(const int32_t* __restrict__ hlist, const int64_t* __restrict__ cstart,
                                                    int B, int* __restrict__ q, int* __restrict__ hpre) {
  __shared__ int carry;
  const int nh = q[64];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nh; b0 += blockDim.x) {
    const int i = b0 + threadIdx.x;
    int v = 0;
    if (i < nh) {
      const int c = hlist[i];
      v = (int)((cstart[c + 1] - cstart[c] + B - 1) / B);
    }
    int64_t tot;
    const int64_t ex = block_excl_scan(v, &tot);
    if (i < nh) hpre[i] = carry + (int)ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += (int)tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    hpre[nh] = carry;
    q[65] = carry;
    q[66] = 0;
  }
}

// Neighbour-set code of a particle: per dimension whether its range reaches the cell below
// (1) or above (2), two bits each.
__device__ __forceinline__ int ppq_code(const PPi& P) {
  int code = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) code |= ((P.lo[d] < 0 ? 1 : 0) | (P.hi[d] > 0 ? 2 : 0)) << (2 * d);
  return code;
}

// The particles of every heavy cell as indices ordered by neighbour-set code, in the
// cell's own index range of hperm (a counting sort per cell; the order within a code is
// arbitrary).  The items of B consecutive entries then hold one or two codes, so that a
// block stages, and a warp computes, only the cells their particles reach.  Each
// particle's sums do not depend on the item or thread that computes them.
__global__ void __launch_bounds__(256) k_ppq_sort_codes(Geo G, const int32_t* __restrict__ hlist,
                                                        const int* __restrict__ q, const int64_t* __restrict__ cstart,
                                                        const int32_t* __restrict__ ires,
                                                        const float4* __restrict__ pfin, int32_t* __restrict__ hperm) {
  __shared__ int cnt[64];
  const int nh = q[64];
  for (int h = blockIdx.x; h < nh; h += gridDim.x) {
    const int c = hlist[h];
    const int64_t s0 = cstart[c], e0 = cstart[c + 1];
    int g[3];
    cell_coords(G, c, g[0], g[1], g[2]);
    const int iapm = ppq_iapm(G, g, ires);
    __syncthreads();  // cnt is free again
    if (threadIdx.x < 64) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int64_t ip = s0 + threadIdx.x; ip < e0; ip += blockDim.x) {
      PPi P;
      P.init(G, g, pfin[ip], iapm);
      atomicAdd(&cnt[ppq_code(P)], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive offsets, two codes per lane
      const int a = cnt[2 * threadIdx.x], b = cnt[2 * threadIdx.x + 1];
      int incl = a + b;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)threadIdx.x >= o) incl += u;
      }
      cnt[2 * threadIdx.x] = incl - a - b;
      cnt[2 * threadIdx.x + 1] = incl - b;
    }
    __syncthreads();
    for (int64_t ip = s0 + threadIdx.x; ip < e0; ip += blockDim.x) {
      PPi P;
      P.init(G, g, pfin[ip], iapm);
      hperm[s0 + atomicAdd(&cnt[ppq_code(P)], 1)] = (int32_t)ip;
    }
  }
}

// Persistent: each block pulls items (B entries of one heavy cell's code-ordered indices)
// from the queue.  The block's particles share their cell, so the candidate cells are the
// 27 around it; a cell that no thread of the block needs is skipped, the others are staged
// in chunks of J, and a warp none of whose particles reaches a cell skips its candidates.
// Pairs in range are deferred: each thread keeps up to PPH_H of them (rv, r2) in its own
// shared-memory column and adds them with PPi::accum, in candidate order, whenever a
// thread of its warp may run out of room; so the force of a pair is evaluated by the lanes
// that have one together, instead of by the whole warp once per lane that has one.
constexpr int PPH_H = 8;   // deferred pairs per thread
constexpr int PPH_U = 4;   // candidates between checks of the deferred count

__host__ __device__ inline size_t ppq_heavy_smem(int B, int J) {
  return (size_t)J * sizeof(float4) + (size_t)PPH_H * B * sizeof(float4);
}

__global__ void k_ppq_heavy(Geo G, const int32_t* __restrict__ hlist, const int* __restrict__ hpre, int* q,
                            const int64_t* __restrict__ cstart, const int32_t* __restrict__ ires,
                            const float4* __restrict__ pfin, const int32_t* __restrict__ hperm, const float* vin,
                            float* vout, const StepDev* __restrict__ sd, int J, float* f2max, float* vmax,
                            unsigned long long* npairs, unsigned long long* ncand, const unsigned* __restrict__ abort) {
  extern __shared__ float4 sj[];  // J candidates, then the deferred pairs [PPH_H][B]
  __shared__ int s_item;
  const int B = blockDim.x;
  float4* const hb = sj + J;
  const bool aborted = abort && *abort;
  const int nh = q[64], nitems = q[65];
  const float mass_scale = sd->pp_mass, v_scale = sd->pp_vscale;
  float f2m = 0.f, av[3] = {0.f, 0.f, 0.f};
  unsigned long long tp = 0, tc = 0;
  for (;;) {
    __syncthreads();  // s_item and sj are free again
    if (threadIdx.x == 0) s_item = aborted ? nitems : atomicAdd(&q[66], 1);
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    // heavy cell of this item: the last h with hpre[h] <= item
    int lo = 0, hi = nh;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (hpre[mid] <= item) lo = mid;
      else hi = mid;
    }
    const int c = hlist[lo];
    const int64_t s0 = cstart[c], e0 = cstart[c + 1];
    const int64_t slot = s0 + (int64_t)(item - hpre[lo]) * B + threadIdx.x;
    const bool live = slot < e0;
    const int64_t ip = live ? (int64_t)hperm[slot] : s0;
    int g[3];
    cell_coords(G, c, g[0], g[1], g[2]);
    PPi P;
    P.init(G, g, pfin[live ? ip : s0], ppq_iapm(G, g, ires));
    int nh = 0;
    auto flush = [&]() {
#pragma unroll 1
      for (int h = 0; h < nh; ++h) {
        const float4 r = hb[h * B + threadIdx.x];
        P.accum(r.x, r.y, r.z, r.w, G.app);
      }
      nh = 0;
    };
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const bool need = live && P.needs(dx, dy, dz);
          if (!__syncthreads_or(need)) continue;  // block-uniform
          const int64_t n = nbr_cell(G, c, P.l, g, dx, dy, dz);
          const int64_t s = cstart[n], e = cstart[n + 1];
          if (need) P.cand += (unsigned)(e - s);
          const float bx = (float)((P.l[0] + dx) * G.rcs), by = (float)((P.l[1] + dy) * G.rcs),
                      bz = (float)((P.l[2] + dz) * G.rcs);
          for (int64_t j0 = s; j0 < e; j0 += J) {
            const int cnt = (int)((e - j0) < (int64_t)J ? (e - j0) : (int64_t)J);
            __syncthreads();
            for (int k = threadIdx.x; k < cnt; k += B) sj[k] = pfin[j0 + k];
            __syncthreads();
            if (__any_sync(0xffffffffu, need))  // warp-uniform
            for (int k0 = 0; k0 < cnt; k0 += PPH_U) {
              if (need) {
                // PPH_U candidates as independent chains (the tail predicated off), their
                // pairs then recorded in candidate order
                float rv[PPH_U][3], r2[PPH_U];
                bool hit[PPH_U];
#pragma unroll
                for (int q = 0; q < PPH_U; ++q) {
                  const bool valid = k0 + q < cnt;
                  const float4 p = sj[valid ? k0 + q : k0];
                  rv[q][0] = __fsub_rn(__fadd_rn(bx, p.x), P.xf[0]);
                  rv[q][1] = __fsub_rn(__fadd_rn(by, p.y), P.xf[1]);
                  rv[q][2] = __fsub_rn(__fadd_rn(bz, p.z), P.xf[2]);
                  r2[q] = sumsq3(rv[q][0], rv[q][1], rv[q][2]);
                  hit[q] = valid && r2[q] > 0.f && r2[q] < P.range2;
                }
#pragma unroll
                for (int q = 0; q < PPH_U; ++q)
                  if (hit[q]) {
                    hb[nh * B + threadIdx.x] = make_float4(rv[q][0], rv[q][1], rv[q][2], r2[q]);
                    ++nh;
                    ++P.pairs;
                  }
              }
              if (__any_sync(0xffffffffu, nh > PPH_H - PPH_U)) flush();
            }
          }
        }
    flush();
    if (live) {
      float a3[3];
      f2m = fmaxf(f2m, ppq_apply(P, ip, vin, vout, mass_scale, v_scale, a3));
#pragma unroll
      for (int d = 0; d < 3; ++d) av[d] = fmaxf(av[d], a3[d]);
      tp += P.pairs;
      tc += P.cand;
    }
  }
  block_max_to(f2m, f2max);
  block_vmax(av, vmax);
  for (int o = 16; o > 0; o >>= 1) {
    tp += __shfl_xor_sync(0xffffffffu, tp, o);
    tc += __shfl_xor_sync(0xffffffffu, tc, o);
  }
  if ((threadIdx.x & 31) == 0 && tp) atomicAdd(npairs, tp);
  if ((threadIdx.x & 31) == 0 && tc) atomicAdd(ncand, tc);
}

// Largest occupancy of the cells [c0, c1) (the autotuner's class key), one atomicMax per
// block.
__global__ void k_ppq_maxcount(const int64_t* __restrict__ cstart, int64_t c0, int64_t c1, int* __restrict__ out) {
  int m = 0;
  for (int64_t c = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += (int64_t)gridDim.x * blockDim.x)
    m = max(m, (int)(cstart[c + 1] - cstart[c]));
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace cube
