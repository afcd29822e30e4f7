// Ghost layers of a run split into z-slabs over ranks (cube_params.nslab > 1), the form
// this library gives buffer_particle.f90's buffer_x / buffer_v (ghost particles copied
// from the neighbouring images before the drift and the kick).  A layer is the ncb coarse
// cell layers next to a slab face (layer_cell in common.cuh); it travels as its per-cell
// counts in slot order and its cells' particles packed in that order, as three arrays
// (ZIPX codes, velocities, ids) one after another in one buffer.  Included by cube_gpu.cu
// after kernels.cuh.
#pragma once
#include "kernels.cuh"

namespace cube {

// Byte offsets of the three arrays of a layer payload of n particles (16-byte aligned).
struct LayerBuf {
  int64_t xo, vo, po, bytes;
};
__host__ __device__ inline LayerBuf layer_buf(int64_t n, int xbytes) {
  LayerBuf b;
  b.xo = 0;
  b.vo = (n * 3 * xbytes + 15) & ~(int64_t)15;
  b.po = b.vo + ((n * 12 + 15) & ~(int64_t)15);
  b.bytes = b.po + n * 8;
  return b;
}

// cnt[slot] = particles of the layer's cell `slot`.
__global__ void k_layer_counts(Geo G, int tz, int lz0, int64_t nlay, const int32_t* __restrict__ rhoc,
                               int32_t* __restrict__ cnt) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nlay) return;
  cnt[s] = rhoc[layer_cell(G, tz, lz0, s)];
}

// The layer's particles into a payload of n particles; pstart: exclusive prefix of the
// slot counts.  One thread per cell, particles in storage order.
__global__ void k_layer_pack(Geo G, int tz, int lz0, int64_t nlay, const int64_t* __restrict__ cstart,
                             const int64_t* __restrict__ pstart, const void* __restrict__ xp,
                             const float* __restrict__ vp, const int64_t* __restrict__ pid, char* __restrict__ buf,
                             int64_t n) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nlay) return;
  const int64_t c = layer_cell(G, tz, lz0, s);
  const int64_t a = cstart[c], m = cstart[c + 1] - a, o = pstart[s];
  const LayerBuf b = layer_buf(n, G.izipx);
  void* bx = buf + b.xo;
  float* bv = reinterpret_cast<float*>(buf + b.vo);
  int64_t* bp = reinterpret_cast<int64_t*>(buf + b.po);
  for (int64_t i = 0; i < m; ++i) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      store_code(bx, G.izipx, 3 * (o + i) + d, load_code(xp, G.izipx, 3 * (a + i) + d));
      bv[3 * (o + i) + d] = vp[3 * (a + i) + d];
    }
    bp[o + i] = pid[a + i];
  }
}

// Counts of a received layer into the cell-count array.
__global__ void k_layer_set_counts(Geo G, int tz, int lz0, int64_t nlay, const int32_t* __restrict__ cnt,
                                   int32_t* __restrict__ rhoc) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nlay) return;
  rhoc[layer_cell(G, tz, lz0, s)] = cnt[s];
}

// A received payload into the particle arrays at the cells' starts.
__global__ void k_layer_unpack(Geo G, int tz, int lz0, int64_t nlay, const int64_t* __restrict__ cstart,
                               const int64_t* __restrict__ pstart, const char* __restrict__ buf, int64_t n,
                               void* __restrict__ xp, float* __restrict__ vp, int64_t* __restrict__ pid) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nlay) return;
  const int64_t c = layer_cell(G, tz, lz0, s);
  const int64_t a = cstart[c], o = pstart[s], m = pstart[s + 1] - o;
  const LayerBuf b = layer_buf(n, G.izipx);
  const void* bx = buf + b.xo;
  const float* bv = reinterpret_cast<const float*>(buf + b.vo);
  const int64_t* bp = reinterpret_cast<const int64_t*>(buf + b.po);
  for (int64_t i = 0; i < m; ++i) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      store_code(xp, G.izipx, 3 * (a + i) + d, load_code(bx, G.izipx, 3 * (o + i) + d));
      vp[3 * (a + i) + d] = bv[3 * (o + i) + d];
    }
    pid[a + i] = bp[o + i];
  }
}

}  // namespace cube
