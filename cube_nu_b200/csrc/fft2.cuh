// Size-specialised FFT passes for the batched Poisson solve.
//
// A length N = R1*R2 transform runs as two register passes over shared memory
// (four-step): with n = R2*n1 + n2 and k = k1 + R1*k2,
//   step 1 (thread n2): R1-point DFT over n1, times w_N^(n2*k1), written in place;
//   step 2 (thread k1): R2-point DFT over n2, written to k1 + R1*k2.
// The R-point DFTs are unrolled in registers, composed recursively from radix 2/3/4
// with inner twiddles read at compile-time indices of a shared table
// tw[j] = e^{-2 pi i j/N} (built on the host in double precision).  With N a template
// parameter every index is strength-reduced; no runtime integer division remains in
// the butterflies.
//
// Passes:
//   k_fx_r2c   : rows of reals, two rows packed as one complex sequence, unpacked into
//                two half spectra (r2c)
//   k_fcol3    : columns (y or z) of the half spectrum, forward / inverse, or forward ->
//                Green multiply -> inverse (z pass); sequences stay in registers
//   k_fx_c2r   : two half-spectrum rows packed as one Hermitian-extended sequence,
//                inverse, real and imaginary parts are the two real rows (c2r)
//   k_fxy3_r2c : for N <= 144 the x and y forward passes of one plane in one block
//   k_fyx3_c2r : its inverse (y then x)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fft.cuh"

namespace cube {
namespace f2 {

// 4-byte asynchronous global -> shared copies (sm_80+ cp.async), used to prefetch the
// Green table while the column data are in flight.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int DIR>
__device__ __forceinline__ float2 twid(const float2* tw, int j) {
  float2 w = tw[j];
  if (DIR > 0) w.y = -w.y;
  return w;
}

template <int R>
struct Split {
  static constexpr int A = (R % 4 == 0 && R != 4) ? 4 : (R % 3 == 0 && R != 3) ? 3 : (R % 2 == 0 && R != 2) ? 2 : R;
  static constexpr int B = R / A;
};

// R-point DFT in registers (sign DIR); inner twiddles from the N-point table.
template <int R, int N, int DIR>
struct DFT {
  static constexpr int A = Split<R>::A, B = Split<R>::B;
  static_assert(N % R == 0, "DFT size must divide the table size");
  __device__ __forceinline__ static void run(float2* v, const float2* tw) {
    float2 tmp[R];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      float2 u[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) u[n1] = v[B * n1 + n2];
      DFT<A, N, DIR>::run(u, tw);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1)
        tmp[k1 * B + n2] = (n2 * k1 == 0) ? u[k1] : cmul(u[k1], twid<DIR>(tw, ((n2 * k1) % R) * (N / R)));
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      float2 w[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) w[n2] = tmp[k1 * B + n2];
      DFT<B, N, DIR>::run(w, tw);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = w[k2];
    }
  }
};

template <int N, int DIR>
struct DFT<1, N, DIR> {
  __device__ __forceinline__ static void run(float2*, const float2*) {}
};

template <int N, int DIR>
struct DFT<2, N, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int N, int DIR>
struct DFT<3, N, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {
    const float s3 = 0.8660254037844386f * (float)DIR;
    const float2 t1 = cadd(v[1], v[2]);
    const float2 d = csub(v[1], v[2]);
    const float2 m0 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    const float2 id = make_float2(-d.y * s3, d.x * s3);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m0, id);
    v[2] = csub(m0, id);
  }
};

template <int N, int DIR>
struct DFT<4, N, DIR> {
  __device__ __forceinline__ static void run(float2* v, const float2*) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
    const float2 jb1 = (DIR < 0) ? make_float2(b1.y, -b1.x) : make_float2(-b1.y, b1.x);
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, jb1);
    v[3] = csub(a1, jb1);
  }
};

// Two-pass sequence transform over shared memory; element e at base[e*se].
template <int N, int R1, int R2, int DIR>
struct Seq {
  static_assert(R1 * R2 == N, "bad factorisation");
  __device__ __forceinline__ static void step1(float2* base, int se, int t, const float2* tw) {
    float2 v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) v[n1] = base[(R2 * n1 + t) * se];
    DFT<R1, N, DIR>::run(v, tw);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) base[(R2 * k1 + t) * se] = (k1 == 0) ? v[0] : cmul(v[k1], twid<DIR>(tw, t * k1));
  }
  __device__ __forceinline__ static void step2_load(const float2* base, int se, int t, float2* w, const float2* tw) {
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) w[n2] = base[(R2 * t + n2) * se];
    DFT<R2, N, DIR>::run(w, tw);
  }
  __device__ __forceinline__ static void step2_store(float2* base, int se, int t, const float2* w) {
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) base[(t + R1 * k2) * se] = w[k2];
  }
};

template <int R1, int R2>
struct TPS {
  static constexpr int T = R1 > R2 ? R1 : R2;  // threads per sequence
};

// Full in-place transform of the sequences handled by this thread group.
// Thread (s, t): s = sequence slot, t in [0, T).  All threads of the block call it.
template <int N, int R1, int R2, int DIR>
__device__ __forceinline__ void seq_transform(float2* base, int se, int t, const float2* tw) {
  using S = Seq<N, R1, R2, DIR>;
  if (t < R2) S::step1(base, se, t, tw);
  __syncthreads();
  float2 w[R2];
  if (t < R1) S::step2_load(base, se, t, w, tw);
  __syncthreads();
  if (t < R1) S::step2_store(base, se, t, w);
  __syncthreads();
}

// Same as seq_transform, for thread groups where some threads have no sequence this
// round (they still take part in the barriers).
template <int N, int R1, int R2, int DIR>
__device__ __forceinline__ void seq_transform_g(float2* base, int se, int t, const float2* tw, bool active) {
  using S = Seq<N, R1, R2, DIR>;
  if (active && t < R2) S::step1(base, se, t, tw);
  __syncthreads();
  float2 w[R2];
  if (active && t < R1) S::step2_load(base, se, t, w, tw);
  __syncthreads();
  if (active && t < R1) S::step2_store(base, se, t, w);
  __syncthreads();
}

// Mesh layouts (both in place, potential written over the input):
//  row-pitched (five-pass sizes): row pitch RP bytes = max(N*rb, (N/2+1)*8), so a real
//    row and its half-spectrum row share bytes (FFTW's in-place r2c layout); plane = N rows;
//  plane-compact (fused sizes): real rows of N, half-spectrum rows of N/2+1 and phi rows of
//    N packed from the start of each plane; plane pitch max(N*N*rb, N*(N/2+1)*8) bytes.
// Kernels take the row pitch (pr real elements, pc complex, pf floats) and the plane pitch
// in the same units (plr, plc, plf).

// ---------------------------------------------------------------------------------
// X pass, r2c.  Block: S packed sequences (2S real rows); blockDim = S*T.  In place:
// the block loads all its rows before writing their spectra.
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2, typename IN>
__global__ void __launch_bounds__(256) k_fx_r2c(const IN* r, float2* c, int64_t nrows, const float2* __restrict__ gtw,
                                                float scale, int pr, int pc) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;
  const int S = blockDim.x / T;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t row0 = (int64_t)blockIdx.x * 2 * S;
  const int nr = (int)min((int64_t)2 * S, nrows - row0);
  for (int i = threadIdx.x; i < 2 * S * N; i += blockDim.x) {
    const int row = i / N, x = i - row * N;
    float f = 0.f;
    if (row < nr) {
      const IN v = r[(row0 + row) * pr + x];
      if (sizeof(IN) == 8) f = (float)((double)(long long)v * 9.094947017729282e-13);  // 2^-40
      else f = (float)v;
      f = __fmul_rn(f, scale);
    }
    reinterpret_cast<float*>(Z + (row >> 1) * N + x)[row & 1] = f;
  }
  __syncthreads();
  const int s = threadIdx.x / T, t = threadIdx.x - s * T;
  seq_transform<N, R1, R2, -1>(Z + s * N, 1, t, tw);
  for (int i = threadIdx.x; i < S * NH; i += blockDim.x) {
    const int q = i / NH, k = i - q * NH;
    if (2 * q >= nr) continue;
    const float2 z = Z[q * N + k];
    const float2 zc = Z[q * N + ((N - k) % N)];
    c[(row0 + 2 * q) * pc + k] = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    if (2 * q + 1 < nr) c[(row0 + 2 * q + 1) * pc + k] = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
  }
}

// ---------------------------------------------------------------------------------
// Column pass with the sequences kept in registers.  Thread (t, col), blockDim = W*T,
// col fastest (coalesced rows of the half spectrum).  Forward (N = R1*R2, n = R2*n1+n2):
// thread t = n2 loads x[R2*n1 + t] straight from global memory, R1-point DFT, twiddle,
// one shared-memory exchange, then thread t = k1 runs the R2-point DFT and holds
// X[t + R1*k2].  The inverse uses the swapped factorisation (n = R1*n1 + n2), whose
// first step needs in thread t exactly the X[t + R1*k2] it already holds, so
// forward -> Green multiply -> inverse costs two exchanges in all.
//   MODE 0: forward, 1: inverse, 2: forward -> multiply by green[kz][y][kx] -> inverse.
// Shared memory: tw[N], exchange slots [N][W] float2, and for MODE 2 the column's Green
// values [N][W] float, prefetched with cp.async at the start.
// ---------------------------------------------------------------------------------
// Launch bounds of the column pass: two blocks per SM where the sequences fit in 64
// registers (or 73 with the 444-thread blocks of N = 144), one block above N = 192.
template <int N>
struct FcolBounds {
  static constexpr int MAXT = (N == 144) ? 448 : 512, MINB = (N <= 192) ? 2 : 1;
};

template <int N, int R1, int R2, int AXIS, int MODE>
__global__ void __launch_bounds__(FcolBounds<N>::MAXT, FcolBounds<N>::MINB) k_fcol3(float2* __restrict__ c, const float* __restrict__ green,
                                                  const float2* __restrict__ gtw, int W, int pc, int64_t plc) {
  constexpr int NH = N / 2 + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* A = sm + N;  // exchange slots, [N][W]
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t line = blockIdx.x;
  const int64_t b = line / N;
  const int o = (int)(line - b * N);
  const int kx0 = blockIdx.y * W;
  const int col = threadIdx.x % W, t = threadIdx.x / W;
  const bool live = kx0 + col < NH;
  const int64_t es = (AXIS == 1) ? pc : plc;
  float2* base = c + b * (int64_t)N * plc + (AXIS == 1 ? (int64_t)o * plc : (int64_t)o * pc) + kx0 + col;
  float2* Ac = A + col;
  float* Gc = reinterpret_cast<float*>(A + (size_t)N * W) + col;  // MODE 2: green[kz] of this column, [N][W]
  if (MODE == 2) {
    if (t < R1 && live) {
      const float* gb = green + (int64_t)o * NH + kx0 + col;  // g[kz][y][kx]
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) cp_async4(Gc + (t + R1 * k2) * W, gb + (int64_t)(t + R1 * k2) * N * NH);
    }
    cp_async_commit();
  }
  __syncthreads();
  if (MODE != 1) {
    // ---- forward: n = R2*n1 + n2 ----
    if (t < R2) {
      float2 v[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = live ? base[(int64_t)(R2 * n1 + t) * es] : make_float2(0.f, 0.f);
      DFT<R1, N, -1>::run(v, tw);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) Ac[(k1 * R2 + t) * W] = (k1 == 0) ? v[0] : cmul(v[k1], twid<-1>(tw, t * k1));
    }
    __syncthreads();
    float2 w[R2];
    if (t < R1) {
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = Ac[(t * R2 + n2) * W];
      DFT<R2, N, -1>::run(w, tw);
    }
    if (MODE == 0) {
      if (t < R1 && live) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) base[(int64_t)(t + R1 * k2) * es] = w[k2];
      }
      return;
    }
    // ---- Green multiply at kz = t + R1*k2 (values this thread prefetched) ----
    cp_async_wait_all();
    if (t < R1 && live) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const float gv = Gc[(t + R1 * k2) * W];
        w[k2] = make_float2(w[k2].x * gv, w[k2].y * gv);
      }
    }
    // ---- inverse, n = R1*n1 + n2 with n2 = t, n1 = k2: first step in registers ----
    if (t < R1) {
      DFT<R2, N, +1>::run(w, tw);
#pragma unroll
      for (int k1 = 1; k1 < R2; ++k1) w[k1] = cmul(w[k1], twid<+1>(tw, t * k1));
    }
    __syncthreads();  // every forward read of the slots is done
    if (t < R1) {
#pragma unroll
      for (int k1 = 0; k1 < R2; ++k1) Ac[(k1 * R1 + t) * W] = w[k1];
    }
    __syncthreads();
    if (t < R2) {
      float2 u[R1];
#pragma unroll
      for (int n2 = 0; n2 < R1; ++n2) u[n2] = Ac[(t * R1 + n2) * W];
      DFT<R1, N, +1>::run(u, tw);
      if (live) {
#pragma unroll
        for (int k2 = 0; k2 < R1; ++k2) base[(int64_t)(t + R2 * k2) * es] = u[k2];
      }
    }
  } else {
    // ---- inverse only, n = R1*n1 + n2: thread t = n2 < R1 loads x[R1*n1 + t] ----
    if (t < R1) {
      float2 w[R2];
#pragma unroll
      for (int n1 = 0; n1 < R2; ++n1) w[n1] = live ? base[(int64_t)(R1 * n1 + t) * es] : make_float2(0.f, 0.f);
      DFT<R2, N, +1>::run(w, tw);
#pragma unroll
      for (int k1 = 0; k1 < R2; ++k1) Ac[(k1 * R1 + t) * W] = (k1 == 0) ? w[0] : cmul(w[k1], twid<+1>(tw, t * k1));
    }
    __syncthreads();
    if (t < R2) {
      float2 u[R1];
#pragma unroll
      for (int n2 = 0; n2 < R1; ++n2) u[n2] = Ac[(t * R1 + n2) * W];
      DFT<R1, N, +1>::run(u, tw);
      if (live) {
#pragma unroll
        for (int k2 = 0; k2 < R1; ++k2) base[(int64_t)(t + R2 * k2) * es] = u[k2];
      }
    }
  }
}

// ---------------------------------------------------------------------------------
// Persistent z pass with Green multiply: the work of k_fcol3<...,2,2> (forward z DFT,
// Green multiply, inverse), one item = W columns of one line (box b, row y), looped over
// by a grid of a few blocks per SM.  The column data and Green values of the next item
// are copied into the other of two shared-memory stages with cp.async while the current
// one is transformed, so the loads stay in flight; the current stage doubles as the
// exchange slots.  Items: it = (b*N + y)*ncg + column group.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__host__ __device__ constexpr int fzs_maxt(int N) { return N <= 192 ? 320 : 512; }

template <int N, int R1, int R2>
__global__ void __launch_bounds__(fzs_maxt(N), (N <= 192 ? 2 : 1)) k_fz_stream(float2* __restrict__ c, const float* __restrict__ green,
                                                            const float2* __restrict__ gtw, int W, int ncg, int pc,
                                                            int64_t plc, int64_t nitems) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* stg = sm + N;                                          // [2][N][W] float2
  float* gst = reinterpret_cast<float*>(stg + (size_t)2 * N * W);  // [2][N][W] float
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int col = threadIdx.x % W, t = threadIdx.x / W;
  const bool thr = t < T;
  auto issue = [&](int64_t it, int st) {  // copy item `it` into stage `st`; always commits a group
    if (it < nitems && thr) {
      const int64_t line = it / ncg;
      const int kx = (int)(it - line * ncg) * W + col;
      if (kx < NH) {
        const int64_t b = line / N;
        const int y = (int)(line - b * N);
        const float2* base = c + b * (int64_t)N * plc + (int64_t)y * pc + kx;
        const float* gb = green + (int64_t)y * NH + kx;
        float2* ds = stg + (size_t)st * N * W + col;
        float* dg = gst + (size_t)st * N * W + col;
#pragma unroll 4
        for (int z = t; z < N; z += T) {
          cp_async8(ds + (size_t)z * W, base + (int64_t)z * plc);
          cp_async4(dg + (size_t)z * W, gb + (int64_t)z * N * NH);
        }
      }
    }
    cp_async_commit();
  };
  int64_t it = blockIdx.x;
  issue(it, 0);
  for (int s = 0; it < nitems; it += gridDim.x, s ^= 1) {
    issue(it + gridDim.x, s ^ 1);
    cp_async_wait_one();  // this thread's copies of item `it` have landed
    __syncthreads();      // and everyone's
    const int64_t line = it / ncg;
    const int kx = (int)(it - line * ncg) * W + col;
    const bool live = thr && kx < NH;
    const int64_t b = line / N;
    const int y = (int)(line - b * N);
    float2* out = c + b * (int64_t)N * plc + (int64_t)y * pc + kx;
    float2* Ac = stg + (size_t)s * N * W + col;
    const float* Gc = gst + (size_t)s * N * W + col;
    // forward, n = R2*n1 + n2: thread t = n2
    float2 v[R1];
    if (thr && t < R2) {
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = live ? Ac[(R2 * n1 + t) * W] : make_float2(0.f, 0.f);
      DFT<R1, N, -1>::run(v, tw);
    }
    __syncthreads();  // the stage's data are in registers; its slots become the exchange
    if (thr && t < R2) {
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) Ac[(k1 * R2 + t) * W] = (k1 == 0) ? v[0] : cmul(v[k1], twid<-1>(tw, t * k1));
    }
    __syncthreads();
    float2 w[R2];
    if (thr && t < R1) {
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) w[n2] = Ac[(t * R2 + n2) * W];
      DFT<R2, N, -1>::run(w, tw);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {  // Green at kz = t + R1*k2
        const float gv = Gc[(t + R1 * k2) * W];
        w[k2] = make_float2(w[k2].x * gv, w[k2].y * gv);
      }
      // inverse, n = R1*n1 + n2 with n2 = t, n1 = k2
      DFT<R2, N, +1>::run(w, tw);
#pragma unroll
      for (int k1 = 1; k1 < R2; ++k1) w[k1] = cmul(w[k1], twid<+1>(tw, t * k1));
    }
    __syncthreads();
    if (thr && t < R1) {
#pragma unroll
      for (int k1 = 0; k1 < R2; ++k1) Ac[(k1 * R1 + t) * W] = w[k1];
    }
    __syncthreads();
    if (thr && t < R2) {
      float2 u[R1];
#pragma unroll
      for (int n2 = 0; n2 < R1; ++n2) u[n2] = Ac[(t * R1 + n2) * W];
      DFT<R1, N, +1>::run(u, tw);
      if (live) {
#pragma unroll
        for (int k2 = 0; k2 < R1; ++k2) out[(int64_t)(t + R2 * k2) * plc] = u[k2];
      }
    }
    __syncthreads();  // this stage is free for the copy issued next iteration
  }
  cp_async_wait_all();
}

// Width and count of the column groups of k_fz_stream: two blocks per SM within
// ~100 KB of shared memory each, at most fzs_maxt(N) threads.
__host__ inline void fz_stream_shape(int N, int T, int& W, int& ncg) {
  const int NH = N / 2 + 1;
  int wmax = (int)((100 * 1024 - 8 * N) / (2 * 12 * N));
  wmax = std::min(wmax, fzs_maxt(N) / T);
  ncg = (NH + wmax - 1) / wmax;
  W = (NH + ncg - 1) / ncg;
}
__host__ inline size_t fz_stream_smem(int N, int W) { return (size_t)N * 8 + (size_t)2 * N * W * 12; }

// Column-block width: the whole half row when it fits one block (<= 512 threads, the
// launch bound), else an even split.
__host__ inline int fcol_width(int N, int T) {
  const int NH = N / 2 + 1;
  const int maxt = (N == 144) ? 448 : 512;  // FcolBounds<N>::MAXT
  for (int nb = 1;; ++nb) {
    const int W = (NH + nb - 1) / nb;
    if (W * T <= maxt && (size_t)W * N * 8 <= 100 * 1024) return W;
  }
}

// ---------------------------------------------------------------------------------
// X' pass, c2r, divided `reps` times by `norm`.  In place (complex rows pc -> real rows pf).
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2>
__global__ void __launch_bounds__(256) k_fx_c2r(const float2* c, float* r, int64_t nrows, const float2* __restrict__ gtw,
                                                float inv, int pc, int pf) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;
  const int S = blockDim.x / T;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t row0 = (int64_t)blockIdx.x * 2 * S;
  const int nr = (int)min((int64_t)2 * S, nrows - row0);
  for (int i = threadIdx.x; i < S * N; i += blockDim.x) {
    const int q = i / N, x = i - q * N;
    float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
    const int k = (x < NH) ? x : N - x;
    if (2 * q < nr) a0 = c[(row0 + 2 * q) * pc + k];
    if (2 * q + 1 < nr) a1 = c[(row0 + 2 * q + 1) * pc + k];
    if (k == 0 || 2 * k == N) { a0.y = 0.f; a1.y = 0.f; }
    if (x >= NH) { a0.y = -a0.y; a1.y = -a1.y; }
    Z[q * N + x] = make_float2(a0.x - a1.y, a0.y + a1.x);
  }
  __syncthreads();
  const int s = threadIdx.x / T, t = threadIdx.x - s * T;
  seq_transform<N, R1, R2, +1>(Z + s * N, 1, t, tw);
  for (int i = threadIdx.x; i < 2 * S * N; i += blockDim.x) {
    const int row = i / N, x = i - row * N;
    if (row >= nr) continue;
    const float2 z = Z[(row >> 1) * N + x];
    float v = (row & 1) ? z.y : z.x;
    r[(row0 + row) * pf + x] = __fmul_rn(v, inv);
  }
}

// ---------------------------------------------------------------------------------
// Plane kernels with register-resident sequences (N <= 144, T = max(R1,R2) <= 16).
// Rows run warp-synchronously: each warp holds two sequences (lanes 0..T-1 and
// 16..16+T-1), loads them straight from global memory and exchanges through a skewed
// slot layout (slot(k1, n2) = k1*R2 + (n2 + k1) mod R2) that is free of bank conflicts
// in both directions.  Columns run as in k_fcol3, W columns by T threads per round.
// The r2c unpack and the c2r Hermitian pack happen on the fly inside the other phase,
// and column results go straight to global memory.
// ---------------------------------------------------------------------------------
constexpr int PLANE3_THREADS = 448;

template <int N>
struct Plane3Sm {
  static constexpr int NH = N / 2 + 1;
  // forward: packed rows Z[N/2][N] + scratch for the self-conjugate columns 0, N/2
  static constexpr size_t FWD = (size_t)(N + (N / 2) * N + 2 * N) * 8;
  // inverse: half spectrum H[N][NH]
  static constexpr size_t INV = (size_t)(N + N * NH) * 8;
};

template <int R1, int R2>
__device__ __forceinline__ int skew(int k1, int n2) {
  int j = n2 + k1;  // < R1 + R2
  if (R1 <= R2) j = (j >= R2) ? j - R2 : j;
  else j = j % R2;
  return k1 * R2 + j;
}

template <int N, int R1, int R2, typename IN>
__global__ void __launch_bounds__(PLANE3_THREADS, 2) k_fxy3_r2c(const IN* __restrict__ r, float2* __restrict__ c,
                                                               const float2* __restrict__ gtw, float scale, int pr,
                                                               int pc, int64_t plr, int64_t plc) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1, NP = N / 2;
  static_assert(T <= 16, "two sequences per warp");
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;  // packed rows, pitch N; then 2N exchange slots for columns 0 and N/2
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t plane = blockIdx.x;
  const IN* rp = r + plane * plr;
  float2* cp = c + plane * plc;
  __syncthreads();
  {  // ---- rows: packed pairs (2p, 2p+1) as re/im ----
    const int lane = threadIdx.x & 31, t = lane & 15;
    const int g = (threadIdx.x >> 5) * 2 + (lane >> 4);
    const int ngr = (blockDim.x >> 5) * 2;
    for (int p0 = 0; p0 < NP; p0 += ngr) {
      const int p = p0 + g;
      const bool act = p < NP;
      float2* Zr = Z + (size_t)(act ? p : 0) * N;
      if (act && t < R2) {
        float2 v[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) {
          const int x = R2 * n1 + t;
          const IN a = rp[(2 * p) * pr + x], b = rp[(2 * p + 1) * pr + x];
          float fa, fb;
          if (sizeof(IN) == 8) {
            fa = (float)((double)(long long)a * 9.094947017729282e-13);
            fb = (float)((double)(long long)b * 9.094947017729282e-13);
          } else {
            fa = (float)a;
            fb = (float)b;
          }
          v[n1] = make_float2(__fmul_rn(fa, scale), __fmul_rn(fb, scale));
        }
        DFT<R1, N, -1>::run(v, tw);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) Zr[skew<R1, R2>(k1, t)] = (k1 == 0) ? v[0] : cmul(v[k1], twid<-1>(tw, t * k1));
      }
      __syncwarp();
      float2 w[R2];
      if (act && t < R1) {
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) w[n2] = Zr[skew<R1, R2>(t, n2)];
        DFT<R2, N, -1>::run(w, tw);
      }
      __syncwarp();
      if (act && t < R1) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) Zr[t + R1 * k2] = w[k2];
      }
      __syncwarp();
    }
  }
  __syncthreads();
  {  // ---- columns kx of the half spectrum, unpacked on the fly ----
    const int W = (NH < (int)blockDim.x / T) ? NH : (int)blockDim.x / T;
    const int col = threadIdx.x % W, t = threadIdx.x / W;
    for (int kx0 = 0; kx0 < NH; kx0 += W) {
      const int kx = kx0 + col;
      const bool act = t < T && kx < NH && col < W;
      const int kc = (N - kx) % N;
      // exchange slot s of column kx (columns kx and N-kx of Z are read only by column
      // kx): slot s < NP at lo + s*st, else at hi + s*st; the self-conjugate columns 0
      // and N/2 use the contiguous scratch S.
      const bool selfc = (kx == 0) || (2 * kx == N);
      const int st = selfc ? 1 : N;
      // offsets from Z (S follows Z): slot s at Z[lo + s*st] for s < NP, else Z[hi + s*st]
      const int64_t lo = selfc ? (int64_t)NP * N + (kx ? N : 0) : (int64_t)kx;
      const int64_t hi = selfc ? lo : (int64_t)kc - (int64_t)NP * N;
      float2 v[R1];
      if (act && t < R2) {
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) {
          const int y = R2 * n1 + t;
          const float2* zr = Z + (size_t)(y >> 1) * N;
          const float2 z = zr[kx], zc = zr[kc];
          v[n1] = (y & 1) ? make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x))
                          : make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
        }
        DFT<R1, N, -1>::run(v, tw);
      }
      __syncthreads();  // all unpack reads of this round are done
      if (act && t < R2) {
        // s = k1*R2 + t < NP exactly when k1 < R1/2 (R1 even) -- resolved per unrolled k1
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
          const int sl = k1 * R2 + t;
          const int64_t b = (k1 * R2 + R2 - 1 < NP) ? lo : ((k1 * R2 >= NP) ? hi : (sl < NP ? lo : hi));
          Z[b + (int64_t)sl * st] = (k1 == 0) ? v[0] : cmul(v[k1], twid<-1>(tw, t * k1));
        }
      }
      __syncthreads();
      if (act && t < R1) {
        float2 w[R2];
        const int s0 = t * R2;
        const bool whole = (s0 + R2 - 1 < NP) || (s0 >= NP);  // R1 even: always
        const int64_t b = (s0 < NP) ? lo : hi;
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) {
          const int sl = s0 + n2;
          w[n2] = Z[(whole ? b : (sl < NP ? lo : hi)) + (int64_t)sl * st];
        }
        DFT<R2, N, -1>::run(w, tw);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) cp[(int64_t)(t + R1 * k2) * pc + kx] = w[k2];
      }
    }
  }
}

template <int N, int R1, int R2>
__global__ void __launch_bounds__(PLANE3_THREADS, 2) k_fyx3_c2r(const float2* __restrict__ c, float* __restrict__ r,
                                                               const float2* __restrict__ gtw, float inv,
                                                               int pc, int pf, int64_t plc, int64_t plf) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1, NP = N / 2;
  static_assert(T <= 16, "two sequences per warp");
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* H = sm + N;  // half spectrum after the inverse y transforms, [N][NH]
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t plane = blockIdx.x;
  const float2* cp = c + plane * plc;
  float* rp = r + plane * plf;
  __syncthreads();
  {  // ---- inverse y transforms of the columns kx, n = R2*n1 + n2 ----
    const int W = (NH < (int)blockDim.x / T) ? NH : (int)blockDim.x / T;
    const int col = threadIdx.x % W, t = threadIdx.x / W;
    for (int kx0 = 0; kx0 < NH; kx0 += W) {
      const int kx = kx0 + col;
      const bool act = t < T && kx < NH && col < W;
      float2* Hc = H + kx;  // column kx: N slots, read and written only by column kx
      if (act && t < R2) {
        float2 v[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) v[n1] = cp[(int64_t)(R2 * n1 + t) * pc + kx];
        DFT<R1, N, +1>::run(v, tw);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) Hc[(k1 * R2 + t) * NH] = (k1 == 0) ? v[0] : cmul(v[k1], twid<+1>(tw, t * k1));
      }
      __syncthreads();
      float2 w[R2];
      if (act && t < R1) {
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) w[n2] = Hc[(t * R2 + n2) * NH];
        DFT<R2, N, +1>::run(w, tw);
      }
      __syncthreads();  // every read of the column's slots is done
      if (act && t < R1) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) Hc[(t + R1 * k2) * NH] = w[k2];
      }
    }
  }
  __syncthreads();
  {  // ---- rows: pack (2p, 2p+1) over the Hermitian extension, inverse x transform ----
    const int lane = threadIdx.x & 31, t = lane & 15;
    const int g = (threadIdx.x >> 5) * 2 + (lane >> 4);
    const int ngr = (blockDim.x >> 5) * 2;
    for (int p0 = 0; p0 < NP; p0 += ngr) {
      const int p = p0 + g;
      const bool act = p < NP;
      float2* H0 = H + (size_t)(act ? 2 * p : 0) * NH;  // rows 2p, 2p+1: 2*NH >= N contiguous slots
      const float2* H1 = H0 + NH;
      float2 v[R1];
      if (act && t < R2) {
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) {
          const int x = R2 * n1 + t;
          const int k = (x < NH) ? x : N - x;
          float2 a0 = H0[k], a1 = H1[k];
          if (k == 0 || 2 * k == N) {
            a0.y = 0.f;
            a1.y = 0.f;
          }
          if (x >= NH) {
            a0.y = -a0.y;
            a1.y = -a1.y;
          }
          v[n1] = make_float2(a0.x - a1.y, a0.y + a1.x);
        }
        DFT<R1, N, +1>::run(v, tw);
      }
      __syncwarp();  // the pack reads of rows 2p, 2p+1 are done
      if (act && t < R2) {
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) H0[skew<R1, R2>(k1, t)] = (k1 == 0) ? v[0] : cmul(v[k1], twid<+1>(tw, t * k1));
      }
      __syncwarp();
      if (act && t < R1) {
        float2 w[R2];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) w[n2] = H0[skew<R1, R2>(t, n2)];
        DFT<R2, N, +1>::run(w, tw);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
          const int x = t + R1 * k2;
          rp[(2 * p) * pf + x] = __fmul_rn(w[k2].x, inv);
          rp[(2 * p + 1) * pf + x] = __fmul_rn(w[k2].y, inv);
        }
      }
      __syncwarp();
    }
  }
}

}  // namespace f2
}  // namespace cube
