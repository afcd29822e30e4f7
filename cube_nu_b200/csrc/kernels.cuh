// Step kernels (header-only, included once by cube_gpu.cu) for one CUBE image on one B200 (sm_100a).
//
// All particle data stays in the reference's order (tile z,y,x; coarse cell z,y,x;
// arrival).  Ghost cells of the reference (buffer_grid.f90, buffer_particle.f90) are
// periodic copies when nn=1, so every kernel reads neighbour cells through periodic
// cell indexing instead of materialised ghost copies.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "fft.cuh"

namespace cube {

// =================================================================================
// Exclusive scan int32 -> int64 (cell starts); out has n+1 entries.
// =================================================================================
static constexpr int SCAN_T = 256, SCAN_I = 8, SCAN_TILE = SCAN_T * SCAN_I;

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v) {
  for (int o = 1; o < 32; o <<= 1) {
    int64_t u = __shfl_up_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns exclusive prefix, total in *tot.
__device__ int64_t block_excl_scan(int64_t v, int64_t* tot) {
  __shared__ int64_t ws[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t inc = warp_incl_scan(v);
  if (lane == 31) ws[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int64_t s = (lane < nw) ? ws[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < nw) ws[lane] = s;
  }
  __syncthreads();
  const int64_t base = (wid > 0) ? ws[wid - 1] : 0;
  *tot = ws[nw - 1];
  __syncthreads();
  return base + inc - v;
}

__global__ void k_scan_tiles(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ tile_sums) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_I;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_I; ++i)
    if (base + i < n) s += in[base + i];
  int64_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(int64_t* __restrict__ sums, int64_t nt) {
  // single block: exclusive scan of nt tile sums in place
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < nt; b0 += blockDim.x) {
    const int64_t i = b0 + threadIdx.x;
    const int64_t v = (i < nt) ? sums[i] : 0;
    int64_t tot;
    const int64_t ex = block_excl_scan(v, &tot);
    if (i < nt) sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[nt] = carry;
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int64_t n, const int64_t* __restrict__ tile_sums,
                             int64_t* __restrict__ out, int64_t ntiles) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_I;
  int64_t v[SCAN_I];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_I; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0;
    s += v[i];
  }
  int64_t tot;
  int64_t ex = block_excl_scan(s, &tot) + tile_sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < SCAN_I; ++i) {
    if (base + i < n) out[base + i] = ex;
    ex += v[i];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_sums[ntiles];
}

inline void exclusive_scan(const int32_t* in, int64_t* out, int64_t n, int64_t* tmp, cudaStream_t s) {
  const int64_t nt = (n + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_tiles<<<(unsigned)nt, SCAN_T, 0, s>>>(in, n, tmp);
  k_scan_sums<<<1, 1024, 0, s>>>(tmp, nt);
  k_scan_apply<<<(unsigned)nt, SCAN_T, 0, s>>>(in, n, tmp, out, nt);
}

// Particle -> storage cell index, from the cell starts.
__global__ void k_fill_pcell(const int64_t* __restrict__ cstart, int64_t ncells, int32_t* __restrict__ pcell) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  for (int64_t i = cstart[c]; i < cstart[c + 1]; ++i) pcell[i] = (int32_t)c;
}

// =================================================================================
// Drift (drift.f90:1-233), bit-exact.
// =================================================================================
// Destination cell, arrival key and count.  The reference scans, per destination
// tile, source cells of the tile's ncb-deep extended region in order
// (ilayer, k, j, i, l) with ilayer=(k-(1-ncb)) mod nlayer (drift.f90:96-115).  The key
// packs that order relative to the destination tile:
//   ilayer:16 | k+ncb-1:8 | j+ncb-1:8 | i+ncb-1:8 | l:24.
// A particle that would move beyond the ghost depth raises CUBE_DEVERR_DRIFT_RANGE (the
// reference stops, drift.f90:64-73) and is kept in its own cell, so the drifted state stays
// a consistent permutation that later kernels can read safely until the host sees the error.
__global__ void k_drift_dest(Geo G, int64_t np, const void* __restrict__ xp, const float* __restrict__ vp,
                             const int32_t* __restrict__ pcell, const int64_t* __restrict__ cstart,
                             const StepDev* __restrict__ sd, int32_t* __restrict__ dest, uint64_t* __restrict__ key,
                             int32_t* __restrict__ count_new, unsigned* err) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  const float dt_mid = sd->dt_mid;
  const int nlayer = sd->nlayer;
  const int c = pcell[ip];
  int g[3];
  cell_coords(G, c, g[0], g[1], g[2]);
  const int64_t l = ip - cstart[c];
  int dn[3];
  bool bad = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int code = load_code(xp, G.izipx, 3 * ip + d);
    const float p = __fmul_rn(dt_mid, vp[3 * ip + d]);
    const double deltax = (double)__fdiv_rn(p, (float)G.rcs);       // drift.f90:57
    const int li = g[d] % G.nt;                                      // i-1 in the source tile
    const double xq = (double)li + zfrac(code, G);                   // drift.f90:59
    const double ig = ceil(__dadd_rn(xq, deltax));                   // drift.f90:63
    if (!(ig >= (double)(1 - 2 * G.ncb) && ig <= (double)(G.nt + 2 * G.ncb))) bad = true;
    dn[d] = bad ? 0 : (int)ig - (li + 1);
  }
  // Source coordinate (i-1) in the destination tile's frame: the ghost copy that lands
  // in the destination's physical cell is the one at (destination - displacement).  When a
  // tile's ghost region wraps onto itself (nc < nt+2ncb) a cell has two copies there and
  // only this one reaches a physical cell.
  int dst[3], rel[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    dst[d] = wrapi(g[d] + dn[d], G.nc);
    const int dloc = dst[d] % G.nt;
    rel[d] = dloc - dn[d];
    if (rel[d] < -G.ncb || rel[d] >= G.nt + G.ncb) bad = true;  // source outside the dest tile's ghost region
  }
  if (bad) {
    set_err(err, CUBE_DEVERR_DRIFT_RANGE);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      dst[d] = g[d];
      rel[d] = g[d] % G.nt;
    }
  }
  const int64_t dc = cell_index(G, dst[0], dst[1], dst[2]);
  if (!owned_cell(G, dc)) {  // lands in another rank's slab, which keeps it
    dest[ip] = -1;
    return;
  }
  const uint64_t kz = (uint64_t)(rel[2] + G.ncb), ky = (uint64_t)(rel[1] + G.ncb), kx = (uint64_t)(rel[0] + G.ncb);
  const uint64_t il = kz % (uint64_t)nlayer;
  // l < 2^24: a cell holds fewer particles than the capacity check on upload allows
  key[ip] = (il << 48) | (kz << 40) | (ky << 32) | (kx << 24) | (uint64_t)(l & 0xffffff);
  dest[ip] = (int32_t)dc;
  atomicAdd(&count_new[dc], 1);
}

__global__ void k_drift_scatter(int64_t np, const int32_t* __restrict__ dest, const uint64_t* __restrict__ key,
                                const int64_t* __restrict__ cstart_new, int32_t* __restrict__ fill,
                                uint64_t* __restrict__ skey, uint32_t* __restrict__ ssrc) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  const int dc = dest[ip];
  if (dc < 0) return;
  const int slot = atomicAdd(&fill[dc], 1);
  const int64_t pos = cstart_new[dc] + slot;
  skey[pos] = key[ip];
  ssrc[pos] = (uint32_t)ip;
}

// Ascending bitonic sort of (key, value) pairs across groups of W lanes (W = 16 or 32);
// lanes pass their index within the group.  Keys are unique; padding lanes hold ~0.
template <int W>
__device__ __forceinline__ void group_bitonic(uint64_t& k, uint32_t& v, int gl) {
#pragma unroll
  for (int size = 2; size <= W; size <<= 1)
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const uint64_t ok = __shfl_xor_sync(0xffffffffu, k, stride);
      const uint32_t ov = __shfl_xor_sync(0xffffffffu, v, stride);
      const bool up = ((gl & size) == 0);
      const bool lower = ((gl & stride) == 0);
      const bool take = lower ? (up ? (ok < k) : (ok > k)) : (up ? (ok > k) : (ok < k));
      if (take) {
        k = ok;
        v = ov;
      }
    }
}

// Two destination cells per warp, one per 16-lane half: segments of <=16 (nearly all at
// 8 particles per cell) are sorted in registers by the half; segments of 17..32 are then
// sorted by the whole warp, one at a time; longer ones are listed for the block sorter.
// Launch (ncells + 1) / 2 warps.
__global__ void k_drift_sort_small(int64_t ncells, const int32_t* __restrict__ count_new,
                                   const int64_t* __restrict__ cstart_new, uint64_t* __restrict__ skey,
                                   uint32_t* __restrict__ ssrc, int32_t* __restrict__ biglist,
                                   int32_t* __restrict__ nbig) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (2 * w >= ncells) return;  // warp-uniform
  const int lane = threadIdx.x & 31;
  const int hl = lane & 15;
  const int64_t c = 2 * w + (lane >> 4);
  const int n = (c < ncells) ? count_new[c] : 0;
  if (n > 32 && hl == 0) biglist[atomicAdd(nbig, 1)] = (int32_t)c;
  const bool small = n > 1 && n <= 16;
  if (__any_sync(0xffffffffu, small)) {
    const int64_t base = small ? cstart_new[c] : 0;
    const bool live = small && hl < n;
    uint64_t k = live ? skey[base + hl] : ~0ull;
    uint32_t v = live ? ssrc[base + hl] : 0u;
    group_bitonic<16>(k, v, hl);
    if (live) {
      skey[base + hl] = k;
      ssrc[base + hl] = v;
    }
  }
  unsigned mid = __ballot_sync(0xffffffffu, n > 16 && n <= 32 && hl == 0);
  while (mid) {
    const int h = __ffs(mid) - 1;
    mid &= mid - 1;
    const int64_t cm = 2 * w + (h >> 4);
    const int nm = count_new[cm];
    const int64_t base = cstart_new[cm];
    uint64_t k = (lane < nm) ? skey[base + lane] : ~0ull;
    uint32_t v = (lane < nm) ? ssrc[base + lane] : 0u;
    group_bitonic<32>(k, v, lane);
    if (lane < nm) {
      skey[base + lane] = k;
      ssrc[base + lane] = v;
    }
  }
}

// Block per long segment: bitonic sort in shared memory (keys are unique), which holds
// max_seg rounded up to a power of two keys and values (drift_sort_smem).  Segments
// longer than max_seg are listed in hugelist for k_drift_rank_huge.
__global__ void k_drift_sort_big(const int32_t* __restrict__ biglist, const int32_t* __restrict__ nbig,
                                 const int32_t* __restrict__ count_new, const int64_t* __restrict__ cstart_new,
                                 uint64_t* __restrict__ skey, uint32_t* __restrict__ ssrc, int max_seg,
                                 int32_t* __restrict__ hugelist, int32_t* __restrict__ nhuge) {
  extern __shared__ uint64_t smk[];
  const int nb = *nbig;
  for (int b = blockIdx.x; b < nb; b += gridDim.x) {  // block-uniform loop over the listed cells
  __syncthreads();  // the previous segment's write-out is done with the shared arrays
  const int c = biglist[b];
  const int n = count_new[c];
  if (n > max_seg) {
    if (threadIdx.x == 0) hugelist[atomicAdd(nhuge, 1)] = c;
    continue;
  }
  int m = 1;
  while (m < n) m <<= 1;  // m <= max_seg rounded up to a power of two: the keys' capacity
  int cap = 1;
  while (cap < max_seg) cap <<= 1;
  uint32_t* smv = reinterpret_cast<uint32_t*>(smk + cap);
  const int64_t base = cstart_new[c];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    smk[i] = (i < n) ? skey[base + i] : ~0ull;
    smv[i] = (i < n) ? ssrc[base + i] : 0u;
  }
  __syncthreads();
  for (int size = 2; size <= m; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = ((i & size) == 0);
          const uint64_t a = smk[i], b = smk[j];
          if ((a > b) == up) {
            smk[i] = b;
            smk[j] = a;
            const uint32_t t = smv[i];
            smv[i] = smv[j];
            smv[j] = t;
          }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    skey[base + i] = smk[i];
    ssrc[base + i] = smv[i];
  }
  }
}

// Dynamic shared memory of k_drift_sort_big for a given max_seg.
inline size_t drift_sort_smem(int max_seg) {
  size_t cap = 1;
  while (cap < (size_t)max_seg) cap <<= 1;
  return cap * 12;
}

// Segments longer than the shared-memory sorter holds (dense halo cores at late times):
// the rank of each key is the number of smaller keys in its segment (keys are unique), so
// it is written straight to its sorted place in (tkey, tsrc); k_drift_copy_huge copies the
// segment back.  Every block walks the listed cells and takes the tiles of 512 elements
// with index = blockIdx.x mod gridDim.x; the segment's keys stream through shared memory in
// chunks.  Quadratic in the segment length (0.3 ms for 5e4 keys), and only such cells run.
constexpr int HUGE_T = 512, HUGE_CHUNK = 4096;
__global__ void __launch_bounds__(HUGE_T) k_drift_rank_huge(const int32_t* __restrict__ hugelist,
                                                            const int32_t* __restrict__ nhuge,
                                                            const int32_t* __restrict__ count_new,
                                                            const int64_t* __restrict__ cstart_new,
                                                            const uint64_t* __restrict__ skey,
                                                            const uint32_t* __restrict__ ssrc,
                                                            uint64_t* __restrict__ tkey, uint32_t* __restrict__ tsrc) {
  __shared__ uint64_t chunk[HUGE_CHUNK];
  const int nh = *nhuge;
  int item = 0;  // running tile index over all listed cells
  for (int h = 0; h < nh; ++h) {
    const int c = hugelist[h];
    const int n = count_new[c];
    const int64_t base = cstart_new[c];
    const int ntile = (n + HUGE_T - 1) / HUGE_T;
    for (int t = 0; t < ntile; ++t, ++item) {
      if (item % gridDim.x != blockIdx.x) continue;  // block-uniform
      const int i = t * HUGE_T + threadIdx.x;
      const bool live = i < n;
      const uint64_t k = live ? skey[base + i] : 0ull;
      int rank = 0;
      for (int j0 = 0; j0 < n; j0 += HUGE_CHUNK) {
        const int cnt = min(HUGE_CHUNK, n - j0);
        __syncthreads();
        for (int j = threadIdx.x; j < cnt; j += HUGE_T) chunk[j] = skey[base + j0 + j];
        __syncthreads();
        if (live)
          for (int j = 0; j < cnt; ++j) rank += chunk[j] < k;
      }
      if (live) {
        tkey[base + rank] = k;
        tsrc[base + rank] = ssrc[base + i];
      }
    }
  }
}

__global__ void k_drift_copy_huge(const int32_t* __restrict__ hugelist, const int32_t* __restrict__ nhuge,
                                  const int32_t* __restrict__ count_new, const int64_t* __restrict__ cstart_new,
                                  const uint64_t* __restrict__ tkey, const uint32_t* __restrict__ tsrc,
                                  uint64_t* __restrict__ skey, uint32_t* __restrict__ ssrc) {
  const int nh = *nhuge;
  for (int h = 0; h < nh; ++h) {
    const int c = hugelist[h];
    const int64_t base = cstart_new[c];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count_new[c];
         i += (int64_t)gridDim.x * blockDim.x) {
      skey[base + i] = tkey[base + i];
      ssrc[base + i] = tsrc[base + i];
    }
  }
}

// New arrays in the sorted order, with the ZIPX update xp+nint(dt_mid*vp/(x_res*ratio_cs))
// in the integer kind (drift.f90:117).
__global__ void k_drift_gather(Geo G, int64_t np, const uint32_t* __restrict__ ssrc, const int32_t* __restrict__ dest,
                               const void* __restrict__ xp, const float* __restrict__ vp,
                               const int64_t* __restrict__ pid, const StepDev* __restrict__ sd, void* __restrict__ xo,
                               float* __restrict__ vo, int64_t* __restrict__ po, int32_t* __restrict__ pcell_o,
                               const int64_t* __restrict__ ntot) {
  // ntot: particles the drift kept (fewer than np when some left this rank's slab)
  const int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= (ntot ? *ntot : np)) return;
  const float dt_mid = sd->dt_mid;
  const int64_t src = ssrc[pos];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float v = vp[3 * src + d];
    const int code = load_code(xp, G.izipx, 3 * src + d);
    const long long dn = llround(__dmul_rn((double)__fmul_rn(dt_mid, v), G.inv_step));
    store_code(xo, G.izipx, 3 * pos + d, (int)(code + (int)dn));
    vo[3 * pos + d] = v;
  }
  if (pid) po[pos] = pid[src];  // null: the ids are permuted later (k_permute_ids)
  pcell_o[pos] = dest[src];
}

// The drift's permutation applied to the particle ids on their own: ids_out[pos] =
// ids_in[ssrc[pos]], for a caller whose ids arrive after the rest of the drift has run.
__global__ void k_permute_ids(int64_t np, const uint32_t* __restrict__ ssrc, const int64_t* __restrict__ ids_in,
                              int64_t* __restrict__ ids_out) {
  const int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pos < np) ids_out[pos] = ids_in[ssrc[pos]];
}

// =================================================================================
// Deposit (particle_mesh.f90:20-109, kick.f90:611-691).
// =================================================================================

template <bool FIXED>
__device__ __forceinline__ void dep_add(void* rho, int64_t i, float w) {
  if (FIXED) {
    atomicAdd(reinterpret_cast<unsigned long long*>(rho) + i, fixed40(w));
  } else {
    atomicAdd(reinterpret_cast<float*>(rho) + i, w);
  }
}

// Mass sums of the deposited density over the physical cells of a level (the reference
// forms them in real(8): particle_mesh.f90:106 testrho, kick.f90:687-688 ptotal), in
// particle units.  The fixed-point form sums the int64 contributions exactly (order
// independent, so deterministic); the FP32 form sums the float weights in FP64.  Warps
// add into one of MASS_SLOTS accumulators picked by block, each on its own 128-byte line
// (MASS_STRIDE words apart), so the atomics spread over many L2 lines; the host adds the
// slots.  A fixed-point slot is 128 bits: word 0 takes the sums, word 1 counts its carries
// (2^40 per particle overflows 64 bits beyond 2^24 particles).
constexpr int MASS_SLOTS = 64, MASS_STRIDE = 16;

__device__ __forceinline__ void warp_sum_to(unsigned long long v, unsigned long long* out) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v && out) {
    unsigned long long* slot = out + (blockIdx.x & (MASS_SLOTS - 1)) * MASS_STRIDE;
    const unsigned long long old = atomicAdd(slot, v);
    if (old + v < old) atomicAdd(slot + 1, 1ull);
  }
}

__device__ __forceinline__ void warp_sum_to(double v, double* out) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0 && out) atomicAdd(out + (blockIdx.x & (MASS_SLOTS - 1)) * MASS_STRIDE, v);
}

// One thread's running mass sum in the arithmetic of its deposit form.
template <bool FIXED>
struct MassAcc {
  using T = typename std::conditional<FIXED, unsigned long long, double>::type;
  T v = 0;
  __device__ __forceinline__ void add(float w) {
    if constexpr (FIXED) v += fixed40(w);
    else v += (double)w;
  }
  // out: MASS_SLOTS accumulators of type T (nullptr: no sum wanted)
  __device__ __forceinline__ void flush(void* out) { warp_sum_to(v, static_cast<T*>(out)); }
};

template <bool FIXED>
__global__ void __launch_bounds__(256, 6) k_deposit_pm1(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                              void* __restrict__ rho, int pr, int64_t pl, void* msum) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  MassAcc<FIXED> mass;
  if (ip < np) {
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  int i2[3];
  float w[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double xpos = (double)g[d] + zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
    i2[d] = tsc_weights(xpos, w[d]);  // xpos*ratio_cs/gridsize with gridsize=ratio_cs is exact
  }
  const int nc = G.nc;
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3) {
    const int z = wrapi(i2[2] - 2 + a3, nc);
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2) {
      const int y = wrapi(i2[1] - 2 + a2, nc);
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        const int x = wrapi(i2[0] - 2 + a1, nc);
        const float ww = __fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]);
        dep_add<FIXED>(rho, (int64_t)z * pl + (int64_t)y * pr + x, ww);
        mass.add(ww);
      }
    }
  }
  }
  mass.flush(msum);
}

// Fixed-point PM1 deposit with the sums of a coarse cell's particles combined in the warp
// first.  A particle of coarse cell g has floor(xpos) = g, so every particle of the cell
// deposits into the same 27 cells; particles are stored cell by cell, so the lanes of a
// warp form runs of equal cells.  For each of the 27 cells the int64 contributions are
// summed over each run (a segmented suffix sum by shuffles) and the run's first lane
// adds the sum with one reduction: about one reduction per cell and run instead of one
// per particle.  Integer sums do not depend on the order, so the density is the one of
// k_deposit_pm1<true>.
__global__ void __launch_bounds__(256) k_deposit_pm1_runs(Geo G, int64_t np, const void* __restrict__ xp,
                                                          const int32_t* __restrict__ pcell,
                                                          unsigned long long* __restrict__ rho, int pr, int64_t pl,
                                                          unsigned long long* msum) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  if ((ip - lane) >= np) return;  // warp-uniform: no live lane in this warp
  const bool live = ip < np;
  const int cell = live ? pcell[ip] : -1 - lane;  // dead lanes form runs of their own
  // run structure: same[k] = lane + 2^k is in this lane's run
  unsigned samebits = 0;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int off = 1 << k;
    const int other = __shfl_down_sync(0xffffffffu, cell, off);
    if (lane + off < 32 && other == cell) samebits |= 1u << k;
  }
  const int prev = __shfl_up_sync(0xffffffffu, cell, 1);
  const bool head = live && (lane == 0 || prev != cell);
  // the longest run decides how many doubling steps are needed
  const unsigned need8 = __ballot_sync(0xffffffffu, samebits & 8u), need16 = __ballot_sync(0xffffffffu, samebits & 16u);
  int g[3] = {0, 0, 0};
  float w[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  if (live) {
    cell_coords(G, cell, g[0], g[1], g[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double xpos = (double)g[d] + zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
      tsc_weights(xpos, w[d]);  // floor(xpos) = g
    }
  }
  const int nc = G.nc;
  unsigned long long mloc = 0;
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3) {
    const int64_t z = (int64_t)wrapi(g[2] - 1 + a3, nc) * pl;
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2) {
      const int64_t y = (int64_t)wrapi(g[1] - 1 + a2, nc) * pr;
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        const float ww = __fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]);
        unsigned long long q = live ? fixed40(ww) : 0ull;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          if (k == 3 && !need8) continue;
          if (k == 4 && !need16) continue;
          const unsigned long long o = __shfl_down_sync(0xffffffffu, q, 1 << k);
          if (samebits & (1u << k)) q += o;
        }
        if (head) {
          atomicAdd(rho + z + y + wrapi(g[0] - 1 + a1, nc), q);
          mloc += q;
        }
      }
    }
  }
  warp_sum_to(mloc, msum);
}

// Candidate tiles along one dimension for a particle with global cell g: its own tile
// and, within ncb of a tile face, the neighbour whose ghost region holds it.
// Writes (tile, local coordinate i-1 in that tile) pairs; returns the count (1 or 2).
__device__ __forceinline__ int tile_cands(const Geo& G, int g, int* t, int* li) {
  const int tt = g / G.nt, l = g - tt * G.nt;
  t[0] = tt;
  li[0] = l;
  // constant slot indices keep the caller's arrays in registers
  const bool lo = l < G.ncb, hi = !lo && l >= G.nt - G.ncb;
  t[1] = wrapi(lo ? tt - 1 : tt + 1, G.nnt);
  li[1] = lo ? l + G.nt : l - G.nt;
  return (lo || hi) ? 2 : 1;
}

// PM2 tile meshes [tile - tile0][ngt^3]; fine index i maps to array i-(1-ngb).
template <bool FIXED>
__global__ void __launch_bounds__(256, 5) k_deposit_pm2(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                              void* __restrict__ rho, int tile0, int ntile, int pr, int64_t pl, void* msum) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  MassAcc<FIXED> mass;
  if (ip < np) {
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  int tc[3][2], lc[3][2], nca[3];
  double f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    nca[d] = tile_cands(G, g[d], tc[d], lc[d]);
    f[d] = zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
  }
  const int ngt = G.ngt;
  const int64_t box = (int64_t)ngt * pl;  // elements per box
  // Candidate loops fully unrolled (at most two per dimension) so the candidate arrays
  // stay in registers.
#pragma unroll
  for (int cz = 0; cz < 2; ++cz)
#pragma unroll
    for (int cy = 0; cy < 2; ++cy)
#pragma unroll
      for (int cx = 0; cx < 2; ++cx) {
        if (cz >= nca[2] || cy >= nca[1] || cx >= nca[0]) continue;
        const int T = (tc[2][cz] * G.nnt + tc[1][cy]) * G.nnt + tc[0][cx];
        if (T < tile0 || T >= tile0 + ntile) continue;
        const int l[3] = {lc[0][cx], lc[1][cy], lc[2][cz]};
        int i2[3];
        float w[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double xpos = ((double)l[d] + f[d]) * (double)G.rcs;  // /gridsize(=1)
          i2[d] = tsc_weights(xpos, w[d]);
        }
        char* base = (char*)rho + (int64_t)(T - tile0) * box * (FIXED ? 8 : 4);
#pragma unroll
        for (int a3 = 0; a3 < 3; ++a3) {
          const int z = i2[2] - 1 + a3 - (1 - G.ngb);
          if (z < 0 || z >= ngt) continue;
#pragma unroll
          for (int a2 = 0; a2 < 3; ++a2) {
            const int y = i2[1] - 1 + a2 - (1 - G.ngb);
            if (y < 0 || y >= ngt) continue;
#pragma unroll
            for (int a1 = 0; a1 < 3; ++a1) {
              const int x = i2[0] - 1 + a1 - (1 - G.ngb);
              if (x < 0 || x >= ngt) continue;
              const float ww = __fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]);
              dep_add<FIXED>(base, (int64_t)z * pl + (int64_t)y * pr + x, ww);
              // physical cells 1..ngp of the tile (array ngb..ngb+ngp-1)
              if ((unsigned)(x - G.ngb) < (unsigned)G.ngp && (unsigned)(y - G.ngb) < (unsigned)G.ngp &&
                  (unsigned)(z - G.ngb) < (unsigned)G.ngp)
                mass.add(ww);
            }
          }
        }
      }
  }
  mass.flush(msum);
}

// Candidate subtiles along one dimension (PM3 nloop=1): own subtile and, in the
// first/last coarse cell of a subtile, the neighbour subtile (possibly in the
// neighbour tile).  Returns count; writes tile, subtile, and local coordinate (i-1)
// in that tile.
__device__ __forceinline__ int sub_cands(const Geo& G, int g, int* t, int* u, int* li) {
  const int tt = g / G.nt, l = g - tt * G.nt;
  const int uu = l / G.ntt, r = l - uu * G.ntt;
  t[0] = tt;
  u[0] = uu;
  li[0] = l;
  // With ntt >= 2 at most one of the two faces is adjacent; constant slot indices keep
  // the caller's arrays in registers.
  const bool lo = r == 0, hi = r == G.ntt - 1;
  if (lo) {
    const bool wrap = uu == 0;
    t[1] = wrap ? wrapi(tt - 1, G.nnt) : tt;
    u[1] = wrap ? G.nns - 1 : uu - 1;
    li[1] = wrap ? l + G.nt : l;
  } else {
    const bool wrap = uu == G.nns - 1;
    t[1] = wrap ? wrapi(tt + 1, G.nnt) : tt;
    u[1] = wrap ? 0 : uu + 1;
    li[1] = wrap ? l - G.nt : l;
  }
  return (lo || hi) ? 2 : 1;
}

__device__ __forceinline__ int subtile_id(const Geo& G, const int t[3], const int u[3]) {
  const int T = (t[2] * G.nnt + t[1]) * G.nnt + t[0];
  return ((T * G.nns + u[2]) * G.nns + u[1]) * G.nns + u[0];
}

// PM3 meshes of one class: slot = box_slot[subtile] (or -1), mesh [slot][nft^3];
// refined index i maps to array i-(1-nfb).
// xpos of kick.f90:628-629, ((l + f) * ratio_cs) / gridsize - u * nfp in real(8), with
// gridsize = real(1/rsf, 4).  For rsf a power of two gridsize is exact and the division
// equals the multiplication by rsf (exact scaling by a power of two).
__device__ __forceinline__ double pm3_xpos(double lf, const Geo& G, double gs, int rsf, int unfp) {
  const double a = lf * (double)G.rcs;
  return (((rsf & (rsf - 1)) == 0) ? a * (double)rsf : a / gs) - (double)unfp;
}

template <bool FIXED>
__global__ void k_deposit_pm3(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                              const int32_t* __restrict__ box_slot, int iapm, void* __restrict__ rho,
                              unsigned* err, int pr, int64_t pl) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  int tc[3][2], uc[3][2], lc[3][2], nca[3];  // at most two candidate subtiles per dimension (ntt >= 2)
  double f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    nca[d] = sub_cands(G, g[d], tc[d], uc[d], lc[d]);
    f[d] = zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
  }
  const int nft = G.nft[iapm], nfp = G.nfp[iapm], nfb = G.nfb[iapm];
  const int64_t box = (int64_t)nft * pl;  // elements per box
  const double gs = (double)(1.f / (float)rsf_of(iapm));  // pm%gridsize, real4
  // Candidate loops fully unrolled (at most two per dimension) so the candidate arrays
  // stay in registers.
#pragma unroll
  for (int cz = 0; cz < 2; ++cz)
#pragma unroll
    for (int cy = 0; cy < 2; ++cy)
#pragma unroll
      for (int cx = 0; cx < 2; ++cx) {
        if (cz >= nca[2] || cy >= nca[1] || cx >= nca[0]) continue;
        const int t[3] = {tc[0][cx], tc[1][cy], tc[2][cz]};
        const int u[3] = {uc[0][cx], uc[1][cy], uc[2][cz]};
        const int slot = box_slot[subtile_id(G, t, u)];
        if (slot < 0) continue;
        const int l[3] = {lc[0][cx], lc[1][cy], lc[2][cz]};
        int i2[3];
        float w[3][3];
        bool oob = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double xpos = pm3_xpos((double)l[d] + f[d], G, gs, rsf_of(iapm), u[d] * nfp);  // kick.f90:628-629
          i2[d] = tsc_weights(xpos, w[d]);
          if (i2[d] - 1 < -nfb || i2[d] + 1 > nfp + nfb + 1) oob = true;
        }
        if (oob) {
          set_err(err, CUBE_DEVERR_DEPOSIT_RANGE);
          continue;
        }
        char* base = (char*)rho + (int64_t)slot * box * (FIXED ? 8 : 4);
#pragma unroll
        for (int a3 = 0; a3 < 3; ++a3) {
          const int z = i2[2] - 1 + a3 - (1 - nfb);
          if (z < 0 || z >= nft) continue;
#pragma unroll
          for (int a2 = 0; a2 < 3; ++a2) {
            const int y = i2[1] - 1 + a2 - (1 - nfb);
            if (y < 0 || y >= nft) continue;
#pragma unroll
            for (int a1 = 0; a1 < 3; ++a1) {
              const int x = i2[0] - 1 + a1 - (1 - nfb);
              if (x < 0 || x >= nft) continue;
              const float ww = __fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]);
              dep_add<FIXED>(base, (int64_t)z * pl + (int64_t)y * pr + x, ww);
            }
          }
        }
      }
}

// PM3 mass over the physical cells of every subtile box (kick.f90:687-688 ptotal), summed
// per particle: for each box the deposit puts the particle in (its own subtile and, in the
// first or last coarse cell of a subtile, the neighbour; each at that box's class), the
// contributions that land in the box's physical cells.  The deposit adds exactly these
// contributions to those cells, so with the fixed-point deposit this is the mesh sum
// itself, exactly; the deposit kernels need no extra work for it.
// A neighbour box of the same class has the own box's weights shifted by whole cells, so
// its physical contributions are the own box's contributions that leave the own physical
// region in its direction: the sum of all 27 own contributions covers both, and
// k_interp_pm3 adds it while it holds the weights.  Only a neighbour of another class (a
// class boundary, rare) needs its own weights: its share of the 27 is replaced by its
// physical contributions at its class (k_mass_pm3).
template <bool FIXED>
__device__ __forceinline__ void mass_box(const Geo& G, int iapm, const double lf[3], const int u[3], int i2[3],
                                         float w[3][3]) {
  const int rsf = rsf_of(iapm), nfp = G.nfp[iapm];
  const double gs = (double)(1.f / (float)rsf);
#pragma unroll
  for (int d = 0; d < 3; ++d) i2[d] = tsc_weights(pm3_xpos(lf[d], G, gs, rsf, u[d] * nfp), w[d]);
}

// direction (-1, 0, +1) of 0-based cell index i relative to the physical range 0..nfp-1
__device__ __forceinline__ int mass_dir(int i, int nfp) { return i < 0 ? -1 : (i >= nfp ? 1 : 0); }

// The class-boundary part: one thread per coarse cell; a cell in a face layer of its
// subtile whose neighbour subtile across that face has another class corrects the own-box
// sums that k_interp_pm3 added for its particles.  Every other cell returns at once.
template <bool FIXED>
__global__ void __launch_bounds__(256) k_mass_pm3(Geo G, const int64_t* __restrict__ cstart,
                                                  const void* __restrict__ xp, const int32_t* __restrict__ ires,
                                                  void* msum) {
  const int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  MassAcc<FIXED> mass;
  int g[3], tc[3][2], uc[3][2], lc[3][2], nca[3] = {1, 1, 1};
  bool any = false;
  int own = 0;
  if (cell < G.ncells && owned_cell(G, cell)) {
    cell_coords(G, cell, g[0], g[1], g[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) nca[d] = sub_cands(G, g[d], tc[d], uc[d], lc[d]);
    if (nca[0] * nca[1] * nca[2] > 1) {
      const int t0[3] = {tc[0][0], tc[1][0], tc[2][0]}, u0[3] = {uc[0][0], uc[1][0], uc[2][0]};
      own = ires[subtile_id(G, t0, u0)];
      for (int cz = 0; cz < nca[2]; ++cz)
        for (int cy = 0; cy < nca[1]; ++cy)
          for (int cx = 0; cx < nca[0]; ++cx) {
            const int t[3] = {tc[0][cx], tc[1][cy], tc[2][cz]}, u[3] = {uc[0][cx], uc[1][cy], uc[2][cz]};
            any |= ires[subtile_id(G, t, u)] != own;
          }
    }
  }
  if (any) {
    const int nfp0 = G.nfp[own];
    const int u0[3] = {uc[0][0], uc[1][0], uc[2][0]};
    for (int64_t ip = cstart[cell]; ip < cstart[cell + 1]; ++ip) {
      double f[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) f[d] = zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
      const double lf0[3] = {(double)lc[0][0] + f[0], (double)lc[1][0] + f[1], (double)lc[2][0] + f[2]};
      int i2[3];
      float w[3][3];
      mass_box<FIXED>(G, own, lf0, u0, i2, w);
      for (int cz = 0; cz < nca[2]; ++cz)
        for (int cy = 0; cy < nca[1]; ++cy)
          for (int cx = 0; cx < nca[0]; ++cx) {
            if (cx + cy + cz == 0) continue;
            const int t[3] = {tc[0][cx], tc[1][cy], tc[2][cz]};
            const int u[3] = {uc[0][cx], uc[1][cy], uc[2][cz]};
            const int nb = ires[subtile_id(G, t, u)];
            if (nb == own) continue;
            int dir[3];
            const int cc[3] = {cx, cy, cz};
#pragma unroll
            for (int d = 0; d < 3; ++d)  // sub_cands: the first coarse cell of a subtile reaches down, the last up
              dir[d] = cc[d] == 0 ? 0 : ((lc[d][0] % G.ntt) == 0 ? -1 : 1);
            // the own contributions in that direction leave the sum ...
            MassAcc<FIXED> sub;
#pragma unroll
            for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
              for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
                for (int a1 = 0; a1 < 3; ++a1)
                  if (mass_dir(i2[0] - 2 + a1, nfp0) == dir[0] && mass_dir(i2[1] - 2 + a2, nfp0) == dir[1] &&
                      mass_dir(i2[2] - 2 + a3, nfp0) == dir[2])
                    sub.add(__fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]));
            mass.v -= sub.v;
            // ... and the neighbour's own physical contributions at its class come in
            const double lf[3] = {(double)lc[0][cx] + f[0], (double)lc[1][cy] + f[1], (double)lc[2][cz] + f[2]};
            int j2[3];
            float v[3][3];
            mass_box<FIXED>(G, nb, lf, u, j2, v);
            const int nfp = G.nfp[nb];
#pragma unroll
            for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
              for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
                for (int a1 = 0; a1 < 3; ++a1)
                  if ((unsigned)(j2[0] - 2 + a1) < (unsigned)nfp && (unsigned)(j2[1] - 2 + a2) < (unsigned)nfp &&
                      (unsigned)(j2[2] - 2 + a3) < (unsigned)nfp)
                    mass.add(__fmul_rn(__fmul_rn(v[0][a1], v[1][a2]), v[2][a3]));
          }
    }
  }
  mass.flush(msum);
}

// Owner-computes form of the fixed-point PM3 deposit: one block per region of
// DEP3_R x DEP3_R x DEP3_RZ cells of one box.  The block sums, in shared memory, the contributions of the
// particles of every coarse cell whose TSC footprint can reach the region, then writes
// every cell of the region (zeros included) with plain stores, so the mesh needs no
// memset and no cell is read back from DRAM.  Cells are written as the float the forward
// FFT would convert the int64 sum to, (float)(q * 2^-40) (unscaled; the FFT multiplies by
// the particle mass), into the float mesh layout: half the bytes of the int64 mesh, and
// the FFT input is bit-identical.  Particle arithmetic is that of
// k_deposit_pm3 (a box's candidate particles are those of coarse cells k = -1..ntt
// around its subtile, with tile-local coordinate l = u*ntt + k), so the int64 sums are
// identical.  Requires at most DEP3_MAXC candidate coarse cells per region (checked on
// the host); the padding of the float layouts is left alone (the FFT never reads it).
constexpr int DEP3_R = 24;   // region extent in x and y (cells)
constexpr int DEP3_RZ = 24;  // region extent in z
constexpr int DEP3_MAXC = 125;
constexpr int DEP3_THREADS = 512;
constexpr int DEP3_MINB = 2;  // blocks per SM
constexpr int DEP3_SPLIT_MAX = 4095;

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Candidate coarse-cell range (box-relative k) along one dimension for region cells
// [o, o+e): TSC footprints fl+nfb-1..fl+nfb+1, one cell of margin for the FP64 rounding
// of xpos.
__device__ __forceinline__ void dep3_krange(int o, int e, int nfb, int ntt, int& klo, int& nk) {
  klo = max(-1, floor_div(o - nfb - 2, nfb));
  const int khi = min(ntt, floor_div(o + e - nfb + 1, nfb));
  nk = khi - klo + 1;
}

__global__ void __launch_bounds__(DEP3_THREADS, DEP3_MINB) k_deposit_pm3_own(Geo G, const void* __restrict__ xp,
                                                                     const int64_t* __restrict__ cstart,
                                                                     const int32_t* __restrict__ box_sub, int iapm,
                                                                     float* __restrict__ rho, unsigned* err,
                                                                     int pr, int64_t pl, int nrx, int nry, int nrz) {
  constexpr int R = DEP3_R, RZ = DEP3_RZ;
  static_assert(R % 2 == 0 && R / 2 <= 16, "a half warp writes one region row");
  extern __shared__ __align__(16) unsigned long long acc[];  // [RZ][R][R]
  __shared__ int64_t cst[DEP3_MAXC];
  __shared__ int ccnt[DEP3_MAXC], ckk[DEP3_MAXC], cpre[DEP3_MAXC + 1];
  const int tid = threadIdx.x;
  const int nft = G.nft[iapm], nfp = G.nfp[iapm], nfb = G.nfb[iapm];
  const int nreg = nrx * nry * nrz;
  const int64_t j = blockIdx.x / nreg;
  const int r = (int)(blockIdx.x - j * nreg);
  const int o[3] = {(r % nrx) * R, ((r / nrx) % nry) * R, (r / (nrx * nry)) * RZ};
  const int e[3] = {min(R, nft - o[0]), min(R, nft - o[1]), min(RZ, nft - o[2])};
  // subtile of this box; -1 pads a class list beyond its count (the slot is never read)
  const int s = box_sub[j];
  if (s < 0) return;
  const int nns3 = G.nns * G.nns * G.nns;
  const int T = s / nns3, f = s - T * nns3;
  const int t[3] = {T % G.nnt, (T / G.nnt) % G.nnt, T / (G.nnt * G.nnt)};
  const int u[3] = {f % G.nns, (f / G.nns) % G.nns, f / (G.nns * G.nns)};
  int klo[3], nk[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) dep3_krange(o[d], e[d], nfb, G.ntt, klo[d], nk[d]);
  const int ncand = nk[0] * nk[1] * nk[2];
  if (ncand > DEP3_MAXC) {  // block-uniform; the host sizes regions so this does not happen
    if (tid == 0) set_err(err, CUBE_DEVERR_DEPOSIT_RANGE);
    return;
  }
  // one thread per candidate coarse cell: its particle range and box-relative k
  if (tid < ncand) {
    const int kx = klo[0] + tid % nk[0], ky = klo[1] + (tid / nk[0]) % nk[1], kz = klo[2] + tid / (nk[0] * nk[1]);
    const int64_t cell = cell_index(G, t[0] * G.nt + u[0] * G.ntt + kx, t[1] * G.nt + u[1] * G.ntt + ky,
                                    t[2] * G.nt + u[2] * G.ntt + kz);
    const int64_t a = cstart[cell];
    cst[tid] = a;
    ccnt[tid] = (int)(cstart[cell + 1] - a);
    ckk[tid] = (kx + 1) | ((ky + 1) << 10) | ((kz + 1) << 20);
  }
  {
    ulonglong2* a2 = reinterpret_cast<ulonglong2*>(acc);
    for (int i = tid; i < R * R * RZ / 2; i += blockDim.x) a2[i] = make_ulonglong2(0ull, 0ull);
  }
  __syncthreads();
  if (tid < 32) {  // prefix of the counts
    int carry = 0;
    for (int b0 = 0; b0 < ncand; b0 += 32) {
      const int i = b0 + tid;
      int incl = (i < ncand) ? ccnt[i] : 0;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if (tid >= off) incl += v;
      }
      if (i < ncand) cpre[i + 1] = carry + incl;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (tid == 0) cpre[0] = 0;
  }
  __syncthreads();
  const int total = cpre[ncand];
  const int rsf = rsf_of(iapm);
  const double gs = (double)(1.f / (float)rsf);  // pm%gridsize, real4
  // Each q = round(w * 2^40) <= 2^40.  With at most DEP3_SPLIT_MAX candidate particles no
  // cell takes more than that many contributions, so the low 20 bits and the rest of q
  // can be summed in the two 32-bit halves of the cell without overflow:
  // sum q = (sum hi << 20) + sum lo.  Denser regions use 64-bit atomics.
  const bool split = total <= DEP3_SPLIT_MAX;
  // the visit loop, instantiated for each summation form (block-uniform choice)
  auto visits = [&](auto split_tag) {
    constexpr bool SPLIT = decltype(split_tag)::value;
    for (int v = tid; v < total; v += blockDim.x) {
      int lo = 0, hi = ncand;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (cpre[mid] <= v) lo = mid;
        else hi = mid;
      }
      const int64_t ip = cst[lo] + (v - cpre[lo]);
      const int kk = ckk[lo];
      const int k[3] = {(kk & 1023) - 1, ((kk >> 10) & 1023) - 1, (kk >> 20) - 1};
      int code[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) code[d] = load_code(xp, G.izipx, 3 * ip + d);
      int i2[3], c0[3];
      float w[3][3];
      bool oob = false, miss = false;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double xpos = pm3_xpos((double)(u[d] * G.ntt + k[d]) + zfrac(code[d], G), G, gs, rsf, u[d] * nfp);
        i2[d] = tsc_weights(xpos, w[d]);  // kick.f90:628-629
        if (i2[d] - 1 < -nfb || i2[d] + 1 > nfp + nfb + 1) oob = true;
        c0[d] = i2[d] + nfb - 2 - o[d];  // region-local cell of the footprint's first weight
        if (c0[d] + 2 < 0 || c0[d] >= e[d]) miss = true;
      }
      if (oob) {
        set_err(err, CUBE_DEVERR_DEPOSIT_RANGE);
        continue;
      }
      if (miss) continue;
#pragma unroll
      for (int a3 = 0; a3 < 3; ++a3) {
        const int z = c0[2] + a3;
        if (z < 0 || z >= e[2]) continue;
#pragma unroll
        for (int a2 = 0; a2 < 3; ++a2) {
          const int y = c0[1] + a2;
          if (y < 0 || y >= e[1]) continue;
#pragma unroll
          for (int a1 = 0; a1 < 3; ++a1) {
            const int x = c0[0] + a1;
            if (x < 0 || x >= e[0]) continue;
            const float ww = __fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]);
            const unsigned long long q = fixed40(ww);
            unsigned long long* cell = &acc[(z * R + y) * R + x];
            if (SPLIT) {
              unsigned* h = reinterpret_cast<unsigned*>(cell);
              atomicAdd(h, (unsigned)(q & 0xfffffull));
              atomicAdd(h + 1, (unsigned)(q >> 20));
            } else {
              atomicAdd(cell, q);
            }
          }
        }
      }
    }
  };
  if (split) visits(std::true_type{});
  else visits(std::false_type{});
  __syncthreads();
  // every cell of the region.  Sums to floats: q * 2^-40 rounded once to FP32 (the int64
  // to float conversion rounds the exact integer, and scaling by 2^-40 is exact), the value
  // the FFT's conversion of the int64 mesh gives.
  auto tofloat = [&](unsigned long long v) {
    if (split) v = ((v >> 32) << 20) + (v & 0xffffffffull);
    return __fmul_rn(__ll2float_rn((long long)v), 9.094947017729282e-13f);  // 2^-40
  };
  float* base = rho + j * (int64_t)nft * pl + (int64_t)o[2] * pl + (int64_t)o[1] * pr + o[0];
  if (e[0] == R && e[1] == R && e[2] == RZ && (pr & 3) == 0 && (pl & 3) == 0 &&
      ((uintptr_t)base & 15) == 0) {
    // a full region (every region of a class-2 box): four cells per 16-byte store, row and
    // plane from compile-time divisions
    constexpr int QX = R / 4;
    static_assert(R % 4 == 0, "rows of whole float4s");
    for (int i = tid; i < RZ * R * QX; i += blockDim.x) {
      const int row = i / QX, qx = i - row * QX;
      const int z = row / R, y = row - z * R;
      const unsigned long long* a = &acc[(z * R + y) * R + 4 * qx];
      const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(a);
      const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(a + 2);
      __stcs(reinterpret_cast<float4*>(base + (int64_t)z * pl + (int64_t)y * pr) + qx,
             make_float4(tofloat(v0.x), tofloat(v0.y), tofloat(v1.x), tofloat(v1.y)));
    }
    return;
  }
  // a partial region: a half warp per row, two cells per 8-byte store (e[0] and the
  // pitches are even).  z = row / e[1] through a float reciprocal: (row + 0.5) / e[1]
  // is at least 0.5/e[1] from an integer, far above the rounding error for row < R*R.
  const int hx = e[0] >> 1, nrow = e[1] * e[2], hl = tid & 15;
  const float inv_e1 = 1.f / (float)e[1];
  for (int row = tid >> 4; row < nrow; row += blockDim.x >> 4) {
    const int z = (int)(((float)row + 0.5f) * inv_e1);
    const int y = row - z * e[1];
    if (hl < hx) {
      const ulonglong2 val = *reinterpret_cast<const ulonglong2*>(&acc[(z * R + y) * R + 2 * hl]);
      const float2 fv = make_float2(tofloat(val.x), tofloat(val.y));
      __stcs(reinterpret_cast<float2*>(base + (int64_t)z * pl + (int64_t)y * pr) + hl, fv);
    }
  }
}

// =================================================================================
// Force from potential (particle_mesh.f90:224-247, kick.f90:839-862) and max |F|^2.
// =================================================================================
__device__ __forceinline__ float grad4(float pm2, float pm1, float pp1, float pp2) {
  const float w0 = (CUBE_W_ALPHA - 1.f) / 4.f, w1 = -CUBE_W_ALPHA / 2.f, w2 = CUBE_W_ALPHA / 2.f,
              w3 = (1.f - CUBE_W_ALPHA) / 4.f;
  float s = __fmul_rn(pm2, w0);
  s = __fadd_rn(s, __fmul_rn(pm1, w1));
  s = __fadd_rn(s, __fmul_rn(pp1, w2));
  s = __fadd_rn(s, __fmul_rn(pp2, w3));
  return s;
}

__device__ __forceinline__ float sumsq3(float a, float b, float c) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}

__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide max of non-negative values; one atomic per block.  Every thread of the
// block must call it (no early returns before it).
__device__ __forceinline__ void block_max_to(float v, float* out) {
  __shared__ float sm[32];
  v = warp_max(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sm[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : 0.f;
    v = warp_max(v);
    if (lane == 0 && v > 0.f) atomic_max_pos(out, v);
  }
}

// PM1: periodic nc^3 phi[z][y][x].  One warp per x-row, grid-stride over rows.
__global__ void k_f2max_periodic(const float* __restrict__ phi, int nc, float* __restrict__ f2out, int pf, int64_t pl) {
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  float v = 0.f;
  const int nrows = nc * nc;
  for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < nrows; row += gridDim.x * wpb) {
    const int z = row / nc, y = row - z * nc;
    const int zm2 = wrapi(z - 2, nc), zm1 = wrapi(z - 1, nc), zp1 = wrapi(z + 1, nc), zp2 = wrapi(z + 2, nc);
    const int ym2 = wrapi(y - 2, nc), ym1 = wrapi(y - 1, nc), yp1 = wrapi(y + 1, nc), yp2 = wrapi(y + 2, nc);
    auto R = [&](int zz, int yy) { return phi + (size_t)zz * pl + (size_t)yy * pf; };
    const float* r0 = R(z, y);
    for (int x = lane; x < nc; x += 32) {
      const int xm2 = wrapi(x - 2, nc), xm1 = wrapi(x - 1, nc), xp1 = wrapi(x + 1, nc), xp2 = wrapi(x + 2, nc);
      const float fx = grad4(r0[xm2], r0[xm1], r0[xp1], r0[xp2]);
      const float fy = grad4(R(z, ym2)[x], R(z, ym1)[x], R(z, yp1)[x], R(z, yp2)[x]);
      const float fz = grad4(R(zm2, y)[x], R(zm1, y)[x], R(zp1, y)[x], R(zp2, y)[x]);
      v = fmaxf(v, sumsq3(fx, fy, fz));
    }
  }
  block_max_to(v, f2out);
}

// f2max over box meshes phi[b] (row pitch pf, plane pitch pl floats; coordinate i is
// array index i - m1phi; physical cells 1..nforce), z stencil in registers.  Block: a 32x32 (x,y) tile of one
// box, 256 threads; thread (lx, ly) owns cells y = 4*ly .. 4*ly+3 at x = lx.  Halo
// planes (36x36) of phi stream through a 4-stage shared-memory ring filled with cp.async,
// three planes ahead of the one being reduced.  From a plane a thread takes one column
// of 8 values (own phi and the y stencils of its 4 cells) and 4 x stencils, 6 loads per
// cell.  Own phi values of the last 5 planes and fx, fy of the last 3 stay in registers,
// so the force at plane zc-2 completes when plane zc arrives.
constexpr int F3_T = 32, F3_P = F3_T + 4, F3_HALO = F3_P * F3_P, F3_LOADS = (F3_HALO + 255) / 256, F3_STAGES = 4;
__device__ __forceinline__ void f3_cp_async4(float* smem, const float* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__global__ void __launch_bounds__(256, 3) k_f2max_box2(const float* __restrict__ phi, int n, int nforce, int m1phi,
                                                       int nbox, float* __restrict__ f2out, int pf, int64_t pl,
                                                       const int32_t* __restrict__ box_sub) {
  __shared__ float pln[F3_STAGES][F3_HALO];
  const int nt = (nforce + F3_T - 1) / F3_T;
  const int tile = blockIdx.x % (nt * nt);
  const int b = blockIdx.x / (nt * nt);
  if (box_sub && box_sub[b] < 0) return;  // padding slot of a class list: block-uniform, nothing to reduce
  const int tx0 = (tile % nt) * F3_T + 1, ty0 = (tile / nt) * F3_T + 1;  // first physical x, y
  const float* pb = phi + (size_t)b * n * pl;
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
  int off[F3_LOADS];
#pragma unroll
  for (int k = 0; k < F3_LOADS; ++k) {
    const int i = threadIdx.x + k * 256;
    off[k] = -2;  // not a halo element of this thread
    if (i < F3_HALO) {
      const int py = i / F3_P, px = i - py * F3_P;
      const int x = tx0 - 2 + px - m1phi, y = ty0 - 2 + py - m1phi;  // array coordinates, >= 0
      off[k] = (x < n && y < n) ? y * pf + x : -1;
      if (off[k] < 0)
#pragma unroll
        for (int st = 0; st < F3_STAGES; ++st) pln[st][i] = 0.f;  // outside the box: zero, never copied
    }
  }
  const int zlast = nforce + 2;
  auto issue = [&](int zc) {  // copy plane zc into its stage; always commits a group
    if (zc <= zlast) {
      const float* pz = pb + (size_t)(zc - m1phi) * pl;
      float* dst = pln[(zc + 1) & (F3_STAGES - 1)];
#pragma unroll
      for (int k = 0; k < F3_LOADS; ++k)
        if (off[k] >= 0) f3_cp_async4(dst + threadIdx.x + k * 256, pz + off[k]);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const bool xin = tx0 + lx <= nforce;
  bool own[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) own[j] = xin && (ty0 + 4 * ly + j <= nforce);
  float P[4][5], FX[4][3], FY[4][3];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
#pragma unroll
    for (int q = 0; q < 5; ++q) P[j][q] = 0.f;
#pragma unroll
    for (int q = 0; q < 3; ++q) FX[j][q] = FY[j][q] = 0.f;
  }
  float v = 0.f;
  issue(-1);
  issue(0);
  issue(1);
  for (int zc = -1; zc <= zlast; ++zc) {
    asm volatile("cp.async.wait_group 2;\n" ::: "memory");  // this thread's copies of plane zc landed
    __syncthreads();  // everyone's copies landed; the stage of plane zc-1 is free again
    issue(zc + 3);
    const float* c = pln[(zc + 1) & (F3_STAGES - 1)];
    // own column: rows 4*ly .. 4*ly+7 of the halo plane at x = lx + 2
    float col[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) col[r] = c[(4 * ly + r) * F3_P + lx + 2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int q = 0; q < 4; ++q) P[j][q] = P[j][q + 1];
      P[j][4] = col[j + 2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        FX[j][q] = FX[j][q + 1];
        FY[j][q] = FY[j][q + 1];
      }
      const float* row = c + (4 * ly + j + 2) * F3_P + lx + 2;
      FX[j][2] = grad4(row[-2], row[-1], row[1], row[2]);
      FY[j][2] = grad4(col[j], col[j + 1], col[j + 3], col[j + 4]);
      if (zc >= 3 && own[j]) {  // plane zc-2 is complete: phi(zc-4..zc) in P, fx, fy in slot 0
        const float fz = grad4(P[j][0], P[j][1], P[j][3], P[j][4]);
        v = fmaxf(v, sumsq3(FX[j][0], FY[j][0], fz));
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  block_max_to(v, f2out);
}

__host__ inline unsigned f2max_box2_grid(int nforce, int nbox) {
  const int nt = (nforce + F3_T - 1) / F3_T;
  return (unsigned)(nt * nt * nbox);
}

// =================================================================================
// Interpolation and kick (particle_mesh.f90:148-217, kick.f90:745-834).  The force
// at each of the 27 TSC cells is differenced from phi on the fly; the values equal
// those of a stored force grid because each uses the same four phi values.
// =================================================================================
// For each component the 27 TSC terms are summed in the reference order
// (i3 outer, i2, i1 inner; kick.f90:789-795); components are independent sums, so
// they are accumulated one after another to keep the loads to 3 x 63.
template <class PhiFn>
__device__ __forceinline__ void tsc_gather_force(const int i2[3], const float w[3][3], PhiFn P, float dv[3]) {
  const int x0 = i2[0] - 1, y0 = i2[1] - 1, z0 = i2[2] - 1;
  // x component: rows of 7 values along x
  float s = 0.f;
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2) {
      float r[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) r[k] = P(x0 - 2 + k, y0 + a2, z0 + a3);
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        const float F = grad4(r[a1], r[a1 + 1], r[a1 + 3], r[a1 + 4]);
        s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(F, w[0][a1]), w[1][a2]), w[2][a3]));
      }
    }
  dv[0] = s;
  // y component: per a3, a 7 (y) x 3 (x) block
  s = 0.f;
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3) {
    float r[7][3];
#pragma unroll
    for (int k = 0; k < 7; ++k)
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) r[k][a1] = P(x0 + a1, y0 - 2 + k, z0 + a3);
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        const float F = grad4(r[a2][a1], r[a2 + 1][a1], r[a2 + 3][a1], r[a2 + 4][a1]);
        s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(F, w[0][a1]), w[1][a2]), w[2][a3]));
      }
  }
  dv[1] = s;
  // z component: the 27 values first (columns of 7 along z), then the ordered sum
  float F2[3][3][3];
#pragma unroll
  for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
    for (int a1 = 0; a1 < 3; ++a1) {
      float r[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) r[k] = P(x0 + a1, y0 + a2, z0 - 2 + k);
#pragma unroll
      for (int a3 = 0; a3 < 3; ++a3) F2[a3][a2][a1] = grad4(r[a3], r[a3 + 1], r[a3 + 3], r[a3 + 4]);
    }
  s = 0.f;
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1)
        s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(F2[a3][a2][a1], w[0][a1]), w[1][a2]), w[2][a3]));
  dv[2] = s;
}

__device__ __forceinline__ void apply_kick(float* vp, int64_t ip, const float dv[3], float a_mid, float dt,
                                           float av[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float v = kick_add(vp[3 * ip + d], dv[d], a_mid, dt);
    vp[3 * ip + d] = v;
    av[d] = fabsf(v);
  }
}

__device__ __forceinline__ void block_vmax(const float av[3], float* vmax) {
  block_max_to(av[0], vmax + 0);
  block_max_to(av[1], vmax + 1);
  block_max_to(av[2], vmax + 2);
}

__global__ void k_interp_pm1(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                             const float* __restrict__ phi, float* __restrict__ vp, const StepDev* __restrict__ sd,
                             int pf, int64_t pl) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  const float a_mid = sd->a_mid, dt = sd->dt;
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  int i2[3];
  float w[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double xpos = (double)g[d] + zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
    i2[d] = tsc_weights(xpos, w[d]);
  }
  const int nc = G.nc;
  // force index i (1-based, periodic) reads phi(i-2..i+2); array index (i-1) mod nc.
  // Wrapped indices of the 7 positions i2-3..i2+3 per dimension, computed once.
  int wx[7], wy[7], wz[7];
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    wx[k] = wrapi(i2[0] - 4 + k, nc);
    wy[k] = wrapi(i2[1] - 4 + k, nc) * pf;
    wz[k] = wrapi(i2[2] - 4 + k, nc) * (int)pl;
  }
  const int x0 = i2[0] - 1, y0 = i2[1] - 1, z0 = i2[2] - 1;
  auto P = [&](int a, int b, int c) { return __ldg(&phi[wz[c - z0 + 2] + wy[b - y0 + 2] + wx[a - x0 + 2]]); };
  float dv[3], av[3];
  tsc_gather_force(i2, w, P, dv);
  apply_kick(vp, ip, dv, a_mid, dt, av);
}

// PM1 force mesh, as potential_to_force builds it before the interpolation
// (particle_mesh.f90:224-247): at every coarse cell j (0-based, periodic) the three
// components grad4(phi(j-2), phi(j-1), phi(j+1), phi(j+2)), with the same FP32
// operations as tsc_gather_force, stored as float4 (fx, fy, fz, 0), x fastest.
__global__ void k_force_pm1(int nc, const float* __restrict__ phi, int pf, int64_t pl, float4* __restrict__ force) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n3 = (int64_t)nc * nc * nc;
  if (i >= n3) return;
  const int x = (int)(i % nc), y = (int)((i / nc) % nc), z = (int)(i / ((int64_t)nc * nc));
  const int64_t row = (int64_t)z * pl + (int64_t)y * pf, xl = (int64_t)z * pl + x;
  const float* ph = phi;
  auto X = [&](int d) { return __ldg(&ph[row + wrapi(x + d, nc)]); };
  auto Y = [&](int d) { return __ldg(&ph[xl + (int64_t)wrapi(y + d, nc) * pf]); };
  auto Z = [&](int d) { return __ldg(&ph[(int64_t)wrapi(z + d, nc) * pl + (int64_t)y * pf + x]); };
  force[i] = make_float4(grad4(X(-2), X(-1), X(1), X(2)), grad4(Y(-2), Y(-1), Y(1), Y(2)),
                         grad4(Z(-2), Z(-1), Z(1), Z(2)), 0.f);
}

// PM1 interpolation + kick from the force mesh: the 27 TSC points of a particle are the
// cells fl-1..fl+1 around its coarse cell; each component is summed in the order of
// tsc_gather_force (a3 outer, a2, a1 inner) with the same products, so the result is
// bit-identical to differencing phi on the fly.
__global__ void k_interp_pm1_force(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                                   const float4* __restrict__ force, float* __restrict__ vp,
                                   const StepDev* __restrict__ sd) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  const float a_mid = sd->a_mid, dt = sd->dt;
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  int i2[3];
  float w[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double xpos = (double)g[d] + zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
    i2[d] = tsc_weights(xpos, w[d]);
  }
  const int nc = G.nc;
  int64_t jx[3], jy[3], jz[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    jx[a] = wrapi(i2[0] - 2 + a, nc);
    jy[a] = (int64_t)wrapi(i2[1] - 2 + a, nc) * nc;
    jz[a] = (int64_t)wrapi(i2[2] - 2 + a, nc) * nc * nc;
  }
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
    for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        const float4 F = __ldg(&force[jz[a3] + jy[a2] + jx[a1]]);
        sx = __fadd_rn(sx, __fmul_rn(__fmul_rn(__fmul_rn(F.x, w[0][a1]), w[1][a2]), w[2][a3]));
        sy = __fadd_rn(sy, __fmul_rn(__fmul_rn(__fmul_rn(F.y, w[0][a1]), w[1][a2]), w[2][a3]));
        sz = __fadd_rn(sz, __fmul_rn(__fmul_rn(__fmul_rn(F.z, w[0][a1]), w[1][a2]), w[2][a3]));
      }
  const float dv[3] = {sx, sy, sz};
  float av[3];
  apply_kick(vp, ip, dv, a_mid, dt, av);
}

__global__ void __launch_bounds__(256, 3) k_interp_pm2(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                             const float* __restrict__ phi, int tile0, int ntile, float* __restrict__ vp,
                             const StepDev* __restrict__ sd, float* vmax, unsigned* err, int pf, int64_t pl) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float a_mid = sd->a_mid, dt = sd->dt;
  float av[3] = {0.f, 0.f, 0.f};
  if (ip < np) {
    int g[3];
    cell_coords(G, pcell[ip], g[0], g[1], g[2]);
    const int T = ((g[2] / G.nt) * G.nnt + g[1] / G.nt) * G.nnt + g[0] / G.nt;
    if (T >= tile0 && T < tile0 + ntile) {
      int i2[3];
      float w[3][3];
      bool oob = false;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double xpos = ((double)(g[d] % G.nt) + zfrac(load_code(xp, G.izipx, 3 * ip + d), G)) * (double)G.rcs;
        i2[d] = tsc_weights(xpos, w[d]);
        if (i2[d] - 1 < 0 || i2[d] + 1 > G.ngp + 1) oob = true;
      }
      if (oob) {
        set_err(err, CUBE_DEVERR_INTERP_RANGE);
      } else {
        const int n = G.ngt, m1 = 1 - G.ngb;
        const float* pb = phi + (size_t)(T - tile0) * n * pl;
        const int ipl = (int)pl;
        auto P = [&](int a, int b, int c) { return __ldg(&pb[(c - m1) * ipl + (b - m1) * pf + (a - m1)]); };
        float dv[3];
        tsc_gather_force(i2, w, P, dv);
        apply_kick(vp, ip, dv, a_mid, dt, av);
      }
    }
  }
  block_vmax(av, vmax);
}

// msum: PM3 mass slots; each particle adds its own box's 27 contributions (the mass sums
// described at k_mass_pm3), in the arithmetic of the deposit form.
template <bool FIXED>
__global__ void __launch_bounds__(256, 3) k_interp_pm3(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                             const float* __restrict__ phi, const int32_t* __restrict__ box_slot, int iapm,
                             float* __restrict__ vp, const StepDev* __restrict__ sd, float* vmax, unsigned* err,
                             int pf, int64_t pl, void* msum) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float a_mid = sd->a_mid, dt = sd->dt;
  float av[3] = {0.f, 0.f, 0.f};
  MassAcc<FIXED> mass;
  if (ip < np) {
    int g[3];
    cell_coords(G, pcell[ip], g[0], g[1], g[2]);
    int t[3], u[3], l[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      t[d] = g[d] / G.nt;
      l[d] = g[d] - t[d] * G.nt;
      u[d] = l[d] / G.ntt;
    }
    const int slot = box_slot[subtile_id(G, t, u)];
    if (slot >= 0) {
      const int nft = G.nft[iapm], nfp = G.nfp[iapm], nfb = G.nfb[iapm];
      const double gs = (double)(1.f / (float)rsf_of(iapm));
      int i2[3];
      float w[3][3];
      bool oob = false;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double xpos = pm3_xpos((double)l[d] + zfrac(load_code(xp, G.izipx, 3 * ip + d), G), G, gs, rsf_of(iapm), u[d] * nfp);
        i2[d] = tsc_weights(xpos, w[d]);
        if (i2[d] - 1 < 0 || i2[d] + 1 > nfp + 1) oob = true;
      }
      if (oob) {
        set_err(err, CUBE_DEVERR_INTERP_RANGE);
      } else {
        const int m1 = 1 - nfb;
        const float* pb = phi + (size_t)slot * nft * pl;
        const int ipl = (int)pl;
        auto P = [&](int a, int b, int c) { return __ldg(&pb[(c - m1) * ipl + (b - m1) * pf + (a - m1)]); };
        float dv[3];
        tsc_gather_force(i2, w, P, dv);
        apply_kick(vp, ip, dv, a_mid, dt, av);
#pragma unroll
        for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
          for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
            for (int a1 = 0; a1 < 3; ++a1) mass.add(__fmul_rn(__fmul_rn(w[0][a1], w[1][a2]), w[2][a3]));
      }
    }
  }
  block_vmax(av, vmax);
  mass.flush(msum);
}

// =================================================================================
// Subtile classes (kick.f90:108-133) and the box slot map of one class.
// =================================================================================
__global__ void k_classify(Geo G, const int32_t* __restrict__ rhoc, int ns3, int32_t* __restrict__ ires,
                           int32_t* __restrict__ napm) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns3) return;
  if (s < G.s0 || s >= G.s1) {  // another rank's subtile: its class arrives by a max-reduction
    ires[s] = 0;
    return;
  }
  const int nns3 = G.nns * G.nns * G.nns;
  const int T = s / nns3, f = s - T * nns3;
  const int tx = T % G.nnt, ty = (T / G.nnt) % G.nnt, tz = T / (G.nnt * G.nnt);
  const int ux = f % G.nns, uy = (f / G.nns) % G.nns, uz = f / (G.nns * G.nns);
  int mx = 0;
  for (int k = 0; k < G.ntt; ++k)
    for (int j = 0; j < G.ntt; ++j)
      for (int i = 0; i < G.ntt; ++i) {
        const int64_t c = cell_index(G, tx * G.nt + ux * G.ntt + i, ty * G.nt + uy * G.ntt + j, tz * G.nt + uz * G.ntt + k);
        mx = max(mx, rhoc[c]);
      }
  const float npc = (float)mx / 64.f;
  const int r = (npc < 24.f) ? 2 : (npc < 114.f) ? 3 : (npc < 320.f) ? 4 : 5;
  ires[s] = r;
  atomicAdd(&napm[r], 1);
}

// Chunk plan of the PM3 boxes: of the subtiles of class c (2..5) in ascending order, the
// first skip[c] are left out and the next cap[c] at most are listed, in chunks of per[c]
// boxes; chunk j of class c is list kbase[c] + j.  The host sizes it (exactly, or with
// headroom for a captured step; skip > 0 lists what a captured step could not hold) and
// the device fills it from ires.
struct PM3Plan {
  int cap[8], per[8], kbase[8], skip[8];
  int nk, per_max;
};

// Class lists on the device (kick.f90:108-138 classes, kick.f90:141-201 order by class):
// the subtiles of class c in ascending order take slots 0, 1, ... of the chunks of c.
// box_sub[k][slot] = subtile (-1 pads unused slots), box_slot[k][s] = slot (-1: not in
// list k); both arrays arrive filled with -1.  *overflow is set when a class has more
// subtiles than skip + capacity (the ones beyond are not listed).  One block of 1024
// threads; thread t owns a contiguous run of subtiles, so ranks follow subtile order.
__global__ void __launch_bounds__(1024) k_build_lists(const int32_t* __restrict__ ires, int ns3, int s_lo, int s_hi,
                                                      PM3Plan pl, int32_t* __restrict__ box_slot,
                                                      int32_t* __restrict__ box_sub, unsigned* __restrict__ overflow) {
  __shared__ int sc[4][1024];
  const int T = blockDim.x, tid = threadIdx.x;
  const int nown = s_hi - s_lo;  // this rank's subtiles [s_lo, s_hi)
  const int per_t = (nown + T - 1) / T;
  const int s0 = s_lo + min(nown, tid * per_t), s1 = s_lo + min(nown, tid * per_t + per_t);
  int cnt[4] = {0, 0, 0, 0};
  for (int s = s0; s < s1; ++s) cnt[(ires[s] - 2) & 3] += 1;
#pragma unroll
  for (int k = 0; k < 4; ++k) sc[k][tid] = cnt[k];
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    int v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = tid >= off ? sc[k][tid - off] : 0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) sc[k][tid] += v[k];
    __syncthreads();
  }
  int r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = sc[k][tid] - cnt[k];
  for (int s = s0; s < s1; ++s) {
    const int c = ires[s], k = (c - 2) & 3;
    const int rank = r[k]++ - pl.skip[c];
    if (rank >= 0 && rank < pl.cap[c]) {
      const int chunk = rank / pl.per[c], slot = rank - chunk * pl.per[c];
      const int64_t kk = pl.kbase[c] + chunk;
      box_slot[kk * ns3 + s] = slot;
      box_sub[kk * pl.per_max + slot] = s;
    }
  }
  if (tid == 0)
    for (int k = 0; k < 4; ++k)
      if (sc[k][T - 1] > pl.skip[k + 2] + pl.cap[k + 2]) *overflow = 1u;
}

// =================================================================================
// PP (kick.f90:376-588).  Each physical particle sums 0<r^2<range^2 pairs over the
// coarse cells its range can reach; equivalent to the reference's PP-cell lists
// (the PP cell 4/rsf fine cells is wider than the range 3.5/rsf).
// =================================================================================
// The softened force law's coefficient (1/35)/apm^2, a constant of apm.
__device__ __forceinline__ float F_ra_coef(float apm) { return __fdiv_rn(__fdiv_rn(1.f, 35.f), __fmul_rn(apm, apm)); }

// F_ra with its coefficient c = F_ra_coef(apm) passed in, for callers that evaluate it for
// one apm many times; the same operations as F_ra.
__device__ __forceinline__ float F_ra_c(float r, float apm, float c) {
  const float ep = __fdiv_rn(2.f * r, apm);
  if (apm == 0.f || ep > 2.f) return __fdiv_rn(1.f, __fmul_rn(r, r));
  const float e2 = ep * ep, e3 = e2 * ep, e4 = e3 * ep, e5 = e4 * ep, e6 = e5 * ep;
  if (ep > 1.f) return c * (12.f * (1.f / e2) - 224.f + 896.f * ep - 840.f * e2 + 224.f * e3 + 70.f * e4 - 48.f * e5 + 7.f * e6);
  if (ep > 0.f) return c * (224.f * ep - 224.f * e3 + 70.f * e4 + 48.f * e5 - 21.f * e6);
  return 0.f;
}

__device__ __forceinline__ float F_ra(float r, float apm) {
  const float ep = __fdiv_rn(2.f * r, apm);
  if (apm == 0.f || ep > 2.f) return __fdiv_rn(1.f, __fmul_rn(r, r));
  return F_ra_c(r, apm, F_ra_coef(apm));
}

// Candidate coordinate (xq in kick.f90:424): ((lq + (u+0.5)*x_res) * ratio_cs) rounded to
// float.  FAST: lq + (u+0.5)*x_res has at most 8*izipx+1+log2|lq| significant bits; when
// that is <= 24 (int8 codes, or int16 codes with |lq| < 128) the sum is exact in FP32 and
// the result equals the FP64 form bit for bit.
template <bool FAST>
__device__ __forceinline__ float pp_xq(const Geo& G, int lq, int code, float xres_f) {
  if (FAST) {
    const float f = __fmul_rn(__fadd_rn((float)((uint32_t)code & G.zmask), 0.5f), xres_f);
    return __fmul_rn(__fadd_rn((float)lq, f), (float)G.rcs);
  }
  return __fmul_rn((float)((double)lq + zfrac(code, G)), (float)G.rcs);
}

template <bool FAST>
__global__ void k_pp(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                     const int64_t* __restrict__ cstart, const int32_t* __restrict__ ires, float* __restrict__ vp,
                     const StepDev* __restrict__ sd, float* f2max, float* vmax,
                     unsigned long long* npairs, unsigned long long* ncand, const unsigned* __restrict__ abort) {
  const int64_t ip0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float mass_scale = sd->pp_mass, v_scale = sd->pp_vscale;
  // abort: the class lists of a captured step were too short; PM3 is finished for the
  // unlisted subtiles afterwards and PP must follow it, so PP leaves vp alone here
  const bool live = ip0 < np && !(abort && *abort) && owned_cell(G, pcell[ip0]);
  const int64_t ip = live ? ip0 : np - 1;
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
  int t[3], u[3], l[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    t[d] = g[d] / G.nt;
    l[d] = g[d] - t[d] * G.nt;
    u[d] = l[d] / G.ntt;
  }
  const int iapm = ires[subtile_id(G, t, u)];
  const float xres_f = (float)G.x_res;  // a power of two
  const float range = __fdiv_rn(3.5f, (float)rsf_of(iapm));  // apm3(iapm)
  const float range2 = __fmul_rn(range, range);
  float xf[3], fin[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double fr = zfrac(load_code(xp, G.izipx, 3 * ip + d), G);
    xf[d] = __fmul_rn((float)((double)l[d] + fr), (float)G.rcs);  // xvec*ratio_cs (kick.f90:424)
    fin[d] = __fmul_rn((float)fr, (float)G.rcs);                  // offset inside the coarse cell, fine units
  }
  int lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = (fin[d] < range) ? -1 : 0;
    hi[d] = ((float)G.rcs - fin[d] < range) ? 1 : 0;
  }
  float acc[3] = {0.f, 0.f, 0.f};
  unsigned long long cnt = 0, cand = 0;
  if (live)
  for (int dz = lo[2]; dz <= hi[2]; ++dz)
    for (int dy = lo[1]; dy <= hi[1]; ++dy)
      for (int dx = lo[0]; dx <= hi[0]; ++dx) {
        const int64_t c = nbr_cell(G, pcell[ip], l, g, dx, dy, dz);
        const int64_t s = cstart[c], e = cstart[c + 1];
        cand += (unsigned long long)(e - s);
        const int lq[3] = {l[0] + dx, l[1] + dy, l[2] + dz};
        for (int64_t q = s; q < e; ++q) {
          float rv[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) rv[d] = __fsub_rn(pp_xq<FAST>(G, lq[d], load_code(xp, G.izipx, 3 * q + d), xres_f), xf[d]);
          const float r2 = sumsq3(rv[0], rv[1], rv[2]);
          if (r2 > 0.f && r2 < range2) {
            const float rm = __fsqrt_rn(r2);
            const float sc = F_ra(rm, G.app) - F_ra(rm, range);
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[d] += __fdiv_rn(rv[d], rm) * sc;
            ++cnt;
          }
        }
      }
  float f1[3], av[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int d = 0; d < 3; ++d) f1[d] = __fmul_rn(acc[d], mass_scale);
  const float f2 = live ? sumsq3(f1[0], f1[1], f1[2]) : 0.f;
  if (live) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float v = __fadd_rn(vp[3 * ip + d], __fmul_rn(f1[d], v_scale));
      vp[3 * ip + d] = v;
      av[d] = fabsf(v);
    }
  }
  block_max_to(f2, f2max);
  block_vmax(av, vmax);
  unsigned long long c = live ? cnt : 0ull, cd = live ? cand : 0ull;
  for (int o = 16; o > 0; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    cd += __shfl_xor_sync(0xffffffffu, cd, o);
  }
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(npairs, c);
  if ((threadIdx.x & 31) == 0 && cd) atomicAdd(ncand, cd);
}

// =================================================================================
// Total momentum (sum of vp over the particles, per component) in FP64, deterministic:
// each block sums a fixed grid-stride share in a fixed order and a shared-memory tree,
// and writes its partial; the host adds the partials in block order.  MOM_BLOCKS blocks.
// =================================================================================
constexpr int MOM_BLOCKS = 592, MOM_THREADS = 256;
__global__ void __launch_bounds__(MOM_THREADS) k_momentum(const float* __restrict__ vp, int64_t np,
                                                          double* __restrict__ partial) {
  __shared__ double sh[3][MOM_THREADS];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * MOM_THREADS + threadIdx.x; i < np; i += (int64_t)gridDim.x * MOM_THREADS) {
    s0 += (double)vp[3 * i];
    s1 += (double)vp[3 * i + 1];
    s2 += (double)vp[3 * i + 2];
  }
  sh[0][threadIdx.x] = s0;
  sh[1][threadIdx.x] = s1;
  sh[2][threadIdx.x] = s2;
  __syncthreads();
  for (int h = MOM_THREADS / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int d = 0; d < 3; ++d) sh[d][threadIdx.x] += sh[d][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < 3) partial[3 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// =================================================================================
// ZIPV int16 velocity codec (utilities/pp_subtile.f90:61 decode, :125 encode), izipv=2:
//   v = tan(pi*vp/(nvbin-1)) / (sqrt(pi/2)/(sigma_vi*vrel_boost))
//   vp = nint((nvbin-1)*atan(sqrt(pi/2)/(sigma_vi*vrel_boost)*v)/pi)
// with nvbin = 2^16 and vrel_boost = 2.5 (parameters.f90:90,135); FP64 as the reference.
// =================================================================================
__device__ __forceinline__ double zipv_scale(float sigma_vi) {
  return sqrt(3.141592653589793 / 2.0) / ((double)sigma_vi * 2.5);
}

__global__ void k_zipv_decode(const int16_t* __restrict__ code, float* __restrict__ v, int64_t n, float sigma_vi) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double arg = 3.141592653589793 * (double)(float)code[i] / (double)65535.f;
  v[i] = (float)(tan(arg) / zipv_scale(sigma_vi));
}

__global__ void k_zipv_encode(const float* __restrict__ v, int16_t* __restrict__ code, int64_t n, float sigma_vi) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = (double)65535.f * atan(zipv_scale(sigma_vi) * (double)v[i]) / 3.141592653589793;
  code[i] = (int16_t)llround(x);
}

// =================================================================================
// int2real (utilities/int2real.f90:68-86): xv(3,np) real(4) = ZIPX offset + cell index in
// coarse-cell units; the real(8) sum is exact, so one rounding to float.
// =================================================================================
__global__ void k_int2real(Geo G, int64_t np, const void* __restrict__ xp, const int32_t* __restrict__ pcell,
                           float* __restrict__ xv) {
  const int64_t ip = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= np) return;
  int g[3];
  cell_coords(G, pcell[ip], g[0], g[1], g[2]);
#pragma unroll
  for (int d = 0; d < 3; ++d)
    xv[3 * ip + d] = __double2float_rn(zfrac(load_code(xp, G.izipx, 3 * ip + d), G) + (double)g[d]);
}

// =================================================================================
// Green's function (Green/Green.f90:1-80) in FP64, stored real32.
// =================================================================================
__global__ void k_green(float* __restrict__ Gk, int n, float apm_soft, float apm_range, float gridsize) {
  const int nh = n / 2 + 1;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)nh * n * n) return;
  const int k1 = (int)(i % nh), k2 = (int)((i / nh) % n), k3 = (int)(i / ((int64_t)nh * n));
  const float inv_n = 1.f / (float)n;
  const double PI = 3.141592653589793;
  auto fs = [&](int k) {  // fftspace(k+1)
    const int m = ((k + 1 + n / 2 - 1) % n) - n / 2;
    return (2.0 * PI) * (double)inv_n * (double)m;
  };
  const double kv[3] = {fs(k1), fs(k2), fs(k3)};
  const float alpha = 4.f / 3.f;
  double Dv[3], ur[3] = {0, 0, 0};
  for (int d = 0; d < 3; ++d) Dv[d] = (double)alpha * sin(kv[d]) + (double)(1.f - alpha) * sin(2 * kv[d]) / 2;
  for (int i3 = -2; i3 <= 2; ++i3)
    for (int i2 = -2; i2 <= 2; ++i2)
      for (int i1 = -2; i1 <= 2; ++i1) {
        const double kn[3] = {kv[0] + 2 * PI * i1, kv[1] + 2 * PI * i2, kv[2] + 2 * PI * i3};
        const double kmag = sqrt(kn[0] * kn[0] + kn[1] * kn[1] + kn[2] * kn[2]);
        if (kmag == 0) continue;  // only k=0, zeroed below
        double prod = 1;
        for (int d = 0; d < 3; ++d) prod *= (kn[d] == 0) ? 1.0 : sin(kn[d] / 2) / (kn[d] / 2);
        const double p2 = prod * prod;
        const double Uk2 = p2 * p2 * p2;
        double y = (double)apm_soft * kmag / 2;
        const double Ss = 12 / (y * y * y * y) * (2 - 2 * cos(y) - y * sin(y));
        double Sr;
        if (apm_range == 0.f) Sr = 0;
        else {
          y = (double)apm_range * kmag / 2;
          Sr = 12 / (y * y * y * y) * (2 - 2 * cos(y) - y * sin(y));
        }
        for (int d = 0; d < 3; ++d) ur[d] += Uk2 * (kn[d] * (Ss * Ss - Sr * Sr) / (kmag * kmag));
      }
  double u2n = 1;
  const double two15 = (double)(2.f / 15.f);
  for (int d = 0; d < 3; ++d) {
    const double s = sin(kv[d] / 2);
    u2n *= 1 - s * s + two15 * s * s * s * s;
  }
  const double num = Dv[0] * ur[0] + Dv[1] * ur[1] + Dv[2] * ur[2];
  const double den = Dv[0] * Dv[0] + Dv[1] * Dv[1] + Dv[2] * Dv[2];
  const float gs2 = gridsize * gridsize;
  double val = (den == 0) ? 0.0 : 4 * PI * num / den / (u2n * u2n) / (double)gs2;
  const int h = n / 2;
  if ((k1 % h == 0) && (k2 % h == 0) && (k3 % h == 0)) val = 0.0;  // Green.f90:71
  Gk[i] = (float)val;
}

// =================================================================================
// Neutrino linear response of the force kernels (kick.f90:23-29; power_nu.f90:179-219
// interp_tf_F, :449-476 nu_correction): tf(k) = interp_tf_F(|k|) * Gk(k) for every mode
// of a Green table, the zero mode set to 1 as nu_correction leaves it.  k of mode
// (i, j, k) (1-based) is (mod(i + n/2, n) - n/2 - 1) * 2 pi / size with `size` the level's
// box side in Mpc/h (box for PM1, box/nnt for PM2, box/nnt/nns for PM3), rounded to real
// as the reference stores kx.  The interpolation is quadratic in log-log through the three
// table points nearest log|k|, in FP32 as the reference computes it.
// =================================================================================
__device__ float nu_interp_tf(const float* __restrict__ klog, const float* __restrict__ tlog, int nb, float kr) {
  const float kn = logf(kr);
  int i1 = 1, i2 = nb;  // 1-based as the reference
  while (i2 - i1 > 1) {
    const int mid = (i1 + i2) / 2;
    if (kn > klog[mid - 1]) i1 = mid;
    else i2 = mid;
  }
  int i3;
  if (kn - klog[i1 - 1] < klog[i2 - 1] - kn) {
    i3 = i2;
    i2 = i1;
    i1 = i1 - 1;
  } else {
    i3 = i2 + 1;
  }
  if (i3 > nb) {
    --i1;
    --i2;
    --i3;
  }
  if (i1 < 1) {  // |k| below the table's second point: the first three points
    i1 = 1;
    i2 = 2;
    i3 = 3;
  }
  const float K1 = klog[i1 - 1], K2 = klog[i2 - 1], K3 = klog[i3 - 1];
  const float T1 = tlog[i1 - 1], T2 = tlog[i2 - 1], T3 = tlog[i3 - 1];
  const float a1 = (T1 - T2) / (K1 - K2);
  const float a2 = (T2 - T3) / (K2 - K3);
  const float k2 = (a1 - a2) / (K1 - K3);
  const float b2 = a1 - k2 * (K1 + K2);
  const float c2 = T1 - k2 * K1 * K1 - b2 * K1;
  return expf(k2 * kn * kn + b2 * kn + c2);
}

__global__ void k_nu_rescale(int n, double size, const float* __restrict__ gk, float* __restrict__ tf,
                             const float* __restrict__ klog, const float* __restrict__ tlog, int nb, float scale) {
  const int nh = n / 2 + 1;
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (int64_t)nh * n * n) return;
  if (nb < 3) {  // no table: the constant (1 - f_nu) of initialize.f90:316-322
    tf[m] = scale * gk[m];
    return;
  }
  const int i = (int)(m % nh) + 1, j = (int)((m / nh) % n) + 1, k = (int)(m / ((int64_t)nh * n)) + 1;
  if (i == 1 && j == 1 && k == 1) {  // zero frequency
    tf[m] = 1.f;
    return;
  }
  const double f = 2.0 * 3.141592653589793 / size;
  const float kx = (float)(((i + n / 2) % n - n / 2 - 1) * f);
  const float ky = (float)(((j + n / 2) % n - n / 2 - 1) * f);
  const float kz = (float)(((k + n / 2) % n - n / 2 - 1) * f);
  const float kr = sqrtf(kx * kx + ky * ky + kz * kz);
  tf[m] = nu_interp_tf(klog, tlog, nb, kr) * gk[m];
}

}  // namespace cube
