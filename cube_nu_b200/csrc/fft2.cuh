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
// Passes (the same five as the generic kernels in fft.cuh):
//   k_fx_r2c : rows of reals, two rows packed as one complex sequence, unpacked into
//              two half spectra (r2c)
//   k_fcol   : columns (y or z) of the half spectrum, forward / inverse, or forward ->
//              Green multiply -> inverse (z pass)
//   k_fx_c2r : two half-spectrum rows packed as one Hermitian-extended sequence,
//              inverse, real and imaginary parts are the two real rows (c2r)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft.cuh"

namespace cube {
namespace f2 {

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

// ---------------------------------------------------------------------------------
// X pass, r2c.  Block: S packed sequences (2S real rows); blockDim = S*T.
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2, typename IN>
__global__ void __launch_bounds__(256) k_fx_r2c(const IN* __restrict__ r, float2* __restrict__ c, int64_t nrows, const float2* __restrict__ gtw,
                         float scale) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;
  const int S = blockDim.x / T;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t row0 = (int64_t)blockIdx.x * 2 * S;
  const int nr = (int)min((int64_t)2 * S, nrows - row0);
  const IN* rp = r + row0 * N;
  for (int i = threadIdx.x; i < 2 * S * N; i += blockDim.x) {
    const int row = i / N, x = i - row * N;
    float f = 0.f;
    if (row < nr) {
      const IN v = rp[i];
      if (sizeof(IN) == 8) f = (float)((double)(long long)v * 9.094947017729282e-13);  // 2^-40
      else f = (float)v;
      f = __fmul_rn(f, scale);
    }
    reinterpret_cast<float*>(Z + (row >> 1) * N + x)[row & 1] = f;
  }
  __syncthreads();
  const int s = threadIdx.x / T, t = threadIdx.x - s * T;
  seq_transform<N, R1, R2, -1>(Z + s * N, 1, t, tw);
  float2* cp = c + row0 * NH;
  for (int i = threadIdx.x; i < S * NH; i += blockDim.x) {
    const int q = i / NH, k = i - q * NH;
    if (2 * q >= nr) continue;
    const float2 z = Z[q * N + k];
    const float2 zc = Z[q * N + ((N - k) % N)];
    cp[(2 * q) * NH + k] = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    if (2 * q + 1 < nr) cp[(2 * q + 1) * NH + k] = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
  }
}

// ---------------------------------------------------------------------------------
// Column pass on the half spectrum c[b][z][y][kx].  MODE 0: forward, 1: inverse,
// 2: forward, times green[kz][ky][kx], inverse (z pass).  AXIS 1: y, 2: z.
// grid.x = b*N + (z for AXIS 1 | y for AXIS 2), grid.y = kx block of W; blockDim = W*T.
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2, int AXIS, int MODE>
__global__ void __launch_bounds__(512) k_fcol(float2* __restrict__ c, const float* __restrict__ green, const float2* __restrict__ gtw, int W) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1, RPT = N / T;  // rows per thread
  static_assert(N % T == 0, "rows must split evenly over the thread group");
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* A = sm + N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t line = blockIdx.x;
  const int64_t b = line / N;
  const int o = (int)(line - b * N);
  const int kx0 = blockIdx.y * W;
  const int col = threadIdx.x % W, t = threadIdx.x / W;  // blockDim = W*T
  const bool live = kx0 + col < NH;
  const int64_t es = (AXIS == 1) ? NH : (int64_t)N * NH;
  float2* base = c + b * (int64_t)N * N * NH + (AXIS == 1 ? (int64_t)o * N * NH : (int64_t)o * NH) + kx0 + col;
  {
    float2 r[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) r[k] = live ? base[(int64_t)(t + k * T) * es] : make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < RPT; ++k) A[(t + k * T) * W + col] = r[k];
  }
  __syncthreads();
  if (MODE == 1) {
    seq_transform<N, R1, R2, +1>(A + col, W, t, tw);
  } else {
    seq_transform<N, R1, R2, -1>(A + col, W, t, tw);
    if (MODE == 2) {
      if (live) {
        const float* gb = green + (int64_t)o * NH + kx0 + col;  // g[kz][y][kx], kz stride N*NH
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          const int e = t + k * T;
          const float gv = __ldg(gb + (int64_t)e * N * NH);
          const float2 v = A[e * W + col];
          A[e * W + col] = make_float2(v.x * gv, v.y * gv);
        }
      }
      __syncthreads();
      seq_transform<N, R1, R2, +1>(A + col, W, t, tw);
    }
  }
  if (live) {
#pragma unroll
    for (int k = 0; k < RPT; ++k) base[(int64_t)(t + k * T) * es] = A[(t + k * T) * W + col];
  }
}

// Column-block width: the whole half row when it fits one block (<= 512 threads, the
// launch bound), else an even split.
__host__ inline int fcol_width(int N, int T) {
  const int NH = N / 2 + 1;
  for (int nb = 1;; ++nb) {
    const int W = (NH + nb - 1) / nb;
    if (W * T <= 512 && (size_t)W * N * 8 <= 100 * 1024) return W;
  }
}

// ---------------------------------------------------------------------------------
// X' pass, c2r, divided `reps` times by `norm`.
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2>
__global__ void __launch_bounds__(256) k_fx_c2r(const float2* __restrict__ c, float* __restrict__ r, int64_t nrows, const float2* __restrict__ gtw,
                         float norm, int reps) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1;
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;
  const int S = blockDim.x / T;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t row0 = (int64_t)blockIdx.x * 2 * S;
  const int nr = (int)min((int64_t)2 * S, nrows - row0);
  const float2* cp = c + row0 * NH;
  for (int i = threadIdx.x; i < S * N; i += blockDim.x) {
    const int q = i / N, x = i - q * N;
    float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
    const int k = (x < NH) ? x : N - x;
    if (2 * q < nr) a0 = cp[(2 * q) * NH + k];
    if (2 * q + 1 < nr) a1 = cp[(2 * q + 1) * NH + k];
    if (k == 0 || 2 * k == N) { a0.y = 0.f; a1.y = 0.f; }
    if (x >= NH) { a0.y = -a0.y; a1.y = -a1.y; }
    Z[q * N + x] = make_float2(a0.x - a1.y, a0.y + a1.x);
  }
  __syncthreads();
  const int s = threadIdx.x / T, t = threadIdx.x - s * T;
  seq_transform<N, R1, R2, +1>(Z + s * N, 1, t, tw);
  float* rp = r + row0 * N;
  for (int i = threadIdx.x; i < 2 * S * N; i += blockDim.x) {
    const int row = i / N, x = i - row * N;
    if (row >= nr) continue;
    const float2 z = Z[(row >> 1) * N + x];
    float v = (row & 1) ? z.y : z.x;
    for (int q = 0; q < reps; ++q) v = __fdiv_rn(v, norm);
    rp[i] = v;
  }
}

}  // namespace f2
}  // namespace cube
