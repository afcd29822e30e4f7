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
// Column pass on the half spectrum c[b][z][y][kx] (row pitch pc).  MODE 0: forward,
// 1: inverse, 2: forward, times green[kz][ky][kx] (dense, pitch N/2+1), inverse (z pass).
// AXIS 1: y, 2: z.  grid.x = b*N + (z for AXIS 1 | y for AXIS 2), grid.y = kx block of W;
// blockDim = W*T.
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2, int AXIS, int MODE>
__global__ void __launch_bounds__(512, 2) k_fcol(float2* __restrict__ c, const float* __restrict__ green,
                                                 const float2* __restrict__ gtw, int W, int pc, int64_t plc) {
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
  const int64_t es = (AXIS == 1) ? pc : plc;
  float2* base = c + b * (int64_t)N * plc + (AXIS == 1 ? (int64_t)o * plc : (int64_t)o * pc) + kx0 + col;
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
// X' pass, c2r, divided `reps` times by `norm`.  In place (complex rows pc -> real rows pf).
// ---------------------------------------------------------------------------------
template <int N, int R1, int R2>
__global__ void __launch_bounds__(256) k_fx_c2r(const float2* c, float* r, int64_t nrows, const float2* __restrict__ gtw,
                                                float norm, int reps, int pc, int pf) {
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
    for (int q = 0; q < reps; ++q) v = __fdiv_rn(v, norm);
    r[(row0 + row) * pf + x] = v;
  }
}

// ---------------------------------------------------------------------------------
// Fused plane passes (one block per z plane; N small enough that a half-spectrum plane
// fits in shared memory).  Forward: load the real plane, r2c along x (rows packed in
// pairs), FFT along y, store the complex plane in place.  Inverse: the reverse.  This
// removes one read and one write of the whole mesh per direction.
// ---------------------------------------------------------------------------------
template <int N>
struct PlaneSm {
  static constexpr int NH = N / 2 + 1, SP = N + 1;  // packed-row pitch (bank padding)
  static constexpr int ELEMS = ((N / 2) * SP > N * NH) ? (N / 2) * SP : N * NH;
  static constexpr size_t BYTES = (size_t)(N + ELEMS) * 8;
};

constexpr int PLANE_THREADS = 512;

template <int N, int R1, int R2, typename IN>
__global__ void __launch_bounds__(PLANE_THREADS, 2) k_fxy_r2c(const IN* r, float2* c, const float2* __restrict__ gtw,
                                                             float scale, int pr, int pc, int64_t plr, int64_t plc) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1, SP = PlaneSm<N>::SP;
  constexpr int NPAIR = N / 2;
  constexpr int KU = (NPAIR * NH + PLANE_THREADS - 1) / PLANE_THREADS;  // unpack items per thread
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t plane = blockIdx.x;  // b*N + z
  const IN* rp = r + plane * plr;
  float2* cp = c + plane * plc;
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
    const int y = i / N, x = i - y * N;
    const IN v = rp[y * pr + x];
    float f;
    if (sizeof(IN) == 8) f = (float)((double)(long long)v * 9.094947017729282e-13);
    else f = (float)v;
    reinterpret_cast<float*>(Z + (y >> 1) * SP + x)[y & 1] = __fmul_rn(f, scale);
  }
  __syncthreads();
  {  // x transforms of the packed rows, G at a time
    constexpr int G = PLANE_THREADS / T;
    const int s = threadIdx.x / T, t = threadIdx.x - s * T;
    for (int p0 = 0; p0 < NPAIR; p0 += G) {
      const int p = p0 + s;
      seq_transform_g<N, R1, R2, -1>(Z + p * SP, 1, t, tw, s < G && p < NPAIR);
    }
  }
  {  // unpack to the half-spectrum plane X[y][kx] (pitch NH), through registers
    float2 k0[KU], k1[KU];
#pragma unroll
    for (int u = 0; u < KU; ++u) {
      const int i = threadIdx.x + u * PLANE_THREADS;
      if (i < NPAIR * NH) {
        const int p = i / NH, k = i - p * NH;
        const float2 z = Z[p * SP + k];
        const float2 zc = Z[p * SP + ((N - k) % N)];
        k0[u] = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
        k1[u] = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < KU; ++u) {
      const int i = threadIdx.x + u * PLANE_THREADS;
      if (i < NPAIR * NH) {
        const int p = i / NH, k = i - p * NH;
        Z[(2 * p) * NH + k] = k0[u];
        Z[(2 * p + 1) * NH + k] = k1[u];
      }
    }
    __syncthreads();
  }
  {  // y transforms of the columns kx (element stride NH), G columns per round
    constexpr int G = PLANE_THREADS / T;
    const int col = threadIdx.x % G, t = threadIdx.x / G;
    for (int k0 = 0; k0 < NH; k0 += G) {
      const int kx = k0 + col;
      seq_transform_g<N, R1, R2, -1>(Z + kx, NH, t, tw, t < T && kx < NH);
    }
  }
  for (int i = threadIdx.x; i < N * NH; i += blockDim.x) {
    const int y = i / NH, k = i - y * NH;
    cp[y * pc + k] = Z[i];
  }
}

template <int N, int R1, int R2>
__global__ void __launch_bounds__(PLANE_THREADS, 2) k_fyx_c2r(const float2* c, float* r, const float2* __restrict__ gtw,
                                                             float norm, int reps, int pc, int pf, int64_t plc,
                                                             int64_t plf) {
  constexpr int T = TPS<R1, R2>::T, NH = N / 2 + 1, SP = PlaneSm<N>::SP;
  constexpr int NPAIR = N / 2;
  constexpr int KP = (NPAIR * N + PLANE_THREADS - 1) / PLANE_THREADS;  // pack items per thread
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* Z = sm + N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = gtw[i];
  const int64_t plane = blockIdx.x;
  const float2* cp = c + plane * plc;
  float* rp = r + plane * plf;
  for (int i = threadIdx.x; i < N * NH; i += blockDim.x) {
    const int y = i / NH, k = i - y * NH;
    Z[i] = cp[y * pc + k];
  }
  __syncthreads();
  {  // inverse y transforms of the columns
    constexpr int G = PLANE_THREADS / T;
    const int col = threadIdx.x % G, t = threadIdx.x / G;
    for (int k0 = 0; k0 < NH; k0 += G) {
      const int kx = k0 + col;
      seq_transform_g<N, R1, R2, +1>(Z + kx, NH, t, tw, t < T && kx < NH);
    }
  }
  {  // pack rows (2p, 2p+1) as X0 + i X1 over the Hermitian extension (c2r convention)
    float2 kp[KP];
#pragma unroll
    for (int u = 0; u < KP; ++u) {
      const int i = threadIdx.x + u * PLANE_THREADS;
      if (i < NPAIR * N) {
        const int p = i / N, x = i - p * N;
        const int k = (x < NH) ? x : N - x;
        float2 a0 = Z[(2 * p) * NH + k], a1 = Z[(2 * p + 1) * NH + k];
        if (k == 0 || 2 * k == N) { a0.y = 0.f; a1.y = 0.f; }
        if (x >= NH) { a0.y = -a0.y; a1.y = -a1.y; }
        kp[u] = make_float2(a0.x - a1.y, a0.y + a1.x);
      }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < KP; ++u) {
      const int i = threadIdx.x + u * PLANE_THREADS;
      if (i < NPAIR * N) {
        const int p = i / N, x = i - p * N;
        Z[p * SP + x] = kp[u];
      }
    }
    __syncthreads();
  }
  {  // inverse x transforms of the packed rows
    constexpr int G = PLANE_THREADS / T;
    const int s = threadIdx.x / T, t = threadIdx.x - s * T;
    for (int p0 = 0; p0 < NPAIR; p0 += G) {
      const int p = p0 + s;
      seq_transform_g<N, R1, R2, +1>(Z + p * SP, 1, t, tw, s < G && p < NPAIR);
    }
  }
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
    const int y = i / N, x = i - y * N;
    const float2 z = Z[(y >> 1) * SP + x];
    float v = (y & 1) ? z.y : z.x;
    for (int q = 0; q < reps; ++q) v = __fdiv_rn(v, norm);
    rp[y * pf + x] = v;
  }
}

}  // namespace f2
}  // namespace cube
