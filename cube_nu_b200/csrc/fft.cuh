// Staged 3D FFT Poisson solve for batches of cubic meshes (replaces FFTW's
// sfftw_plan_dft_r2c_3d / c2r_3d of cubefft.f90:21-37 and the pencil FFT of
// pencil_fft.f90:23-79 for one GPU).
//
// Layout: real mesh r[b][z][y][x] (x fastest, n per side), half spectrum
// c[b][z][y][kx] with kx in [0, n/2], as FFTW's r2c output in Fortran order.
// Five passes, each one read and one write of the mesh:
//   X  : r2c along x per row      (input scale: mass_p_cdm, fixed-point -> float)
//   Y  : complex FFT along y      (forward)
//   Z  : complex FFT along z, times the real Green table, inverse FFT along z
//   Y' : inverse along y
//   X' : c2r along x, divided by n^3 (phi=phi/real(nwork)**3, kick.f90:846)
// Each 1D transform runs in shared memory as a Stockham autosort FFT with radix
// 4/2/3 stages; twiddles come from a per-size table e^{-2 pi i k/n} built on the host
// in double precision.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cube {

struct FFTDesc {
  int n;
  int nrad;
  int8_t rad[16];
  const float2* tw;  // device, n entries of e^{-2 pi i k/n}
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Batched Stockham FFT in shared memory.  Sequence s, element e at
// buf[s*sb + e*se].  SFAST selects the thread mapping (sequence index fastest when
// the sequences are interleaved, sb==1).  dir=-1 forward, +1 backward.  Returns the
// buffer holding the result.
template <bool SFAST>
__device__ float2* fft_smem(float2* a, float2* b, int n, int nb, int sb, int se, const float2* tw,
                            const FFTDesc& D, int dir) {
  float2* in = a;
  float2* out = b;
  int Ns = 1;
  const float s3 = 0.8660254037844386f * (float)dir;  // sin(2 pi/3) with the transform sign
  for (int st = 0; st < D.nrad; ++st) {
    const int R = D.rad[st];
    const int m = n / R;
    const int total = nb * m;
    const int tws = n / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      int s, j;
      if (SFAST) { s = t % nb; j = t / nb; }
      else { j = t % m; s = t / m; }
      const int jm = j % Ns;
      float2 v[4];
      const float2* src = in + s * sb;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (r < R) v[r] = src[(j + r * m) * se];
#pragma unroll
      for (int r = 1; r < 4; ++r)
        if (r < R) {
          float2 w = tw[r * jm * tws];
          if (dir > 0) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
      float2 y[4];
      if (R == 4) {
        const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        const float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
        // (dir * i) * b1
        const float2 jb1 = (dir < 0) ? make_float2(b1.y, -b1.x) : make_float2(-b1.y, b1.x);
        y[0] = cadd(a0, b0);
        y[2] = csub(a0, b0);
        y[1] = cadd(a1, jb1);
        y[3] = csub(a1, jb1);
      } else if (R == 2) {
        y[0] = cadd(v[0], v[1]);
        y[1] = csub(v[0], v[1]);
      } else {  // R == 3
        const float2 t1 = cadd(v[1], v[2]);
        const float2 d = csub(v[1], v[2]);
        const float2 m0 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
        const float2 id = make_float2(-d.y * s3, d.x * s3);
        y[0] = cadd(v[0], t1);
        y[1] = cadd(m0, id);
        y[2] = csub(m0, id);
      }
      const int idxD = (j / Ns) * Ns * R + jm;
      float2* dst = out + s * sb;
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (r < R) dst[(idxD + r * Ns) * se] = y[r];
    }
    __syncthreads();
    float2* tmp = in;
    in = out;
    out = tmp;
    Ns *= R;
  }
  return in;
}

// ---- X pass: real rows -> half spectrum.  IN = float (plain) or long long (fixed point).
template <typename IN>
__global__ void k_fft_x_r2c(const IN* r, float2* c, int64_t nrows, FFTDesc D, int rpb, float scale, int pr, int pc) {
  extern __shared__ float2 sm[];
  const int n = D.n, nh = n / 2 + 1;
  float2* tw = sm;
  float2* a = sm + n;
  float2* b = a + rpb * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = D.tw[i];
  const int64_t row0 = (int64_t)blockIdx.x * rpb;
  const int nr = (int)min((int64_t)rpb, nrows - row0);
  for (int t = threadIdx.x; t < nr * n; t += blockDim.x) {
    const int rr = t / n, x = t - rr * n;
    const IN v = r[(row0 + rr) * pr + x];
    float f;
    if (sizeof(IN) == 8) f = (float)((double)(long long)v * 9.094947017729282e-13);  // 2^-40
    else f = (float)v;
    a[t] = make_float2(__fmul_rn(f, scale), 0.f);
  }
  __syncthreads();
  float2* res = fft_smem<false>(a, b, n, nr, n, 1, tw, D, -1);
  for (int t = threadIdx.x; t < nr * nh; t += blockDim.x) {
    const int rr = t / nh, x = t - rr * nh;
    c[(row0 + rr) * pc + x] = res[rr * n + x];
  }
}

// ---- Y pass (forward or inverse) on c[b][z][y][kx]; grid = (b*n+z, kx block).
__global__ void k_fft_y(float2* __restrict__ c, FFTDesc D, int W, int dir, int pc, int64_t plc) {
  extern __shared__ float2 sm[];
  const int n = D.n, nh = n / 2 + 1;
  float2* tw = sm;
  float2* a = sm + n;
  float2* b = a + W * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = D.tw[i];
  const int64_t bz = blockIdx.x;  // b*n + z
  const int kx0 = blockIdx.y * W;
  const int wv = min(W, nh - kx0);
  float2* base = c + bz * plc + kx0;
  for (int t = threadIdx.x; t < n * W; t += blockDim.x) {
    const int y = t / W, q = t - y * W;
    a[y * W + q] = (q < wv) ? base[(int64_t)y * pc + q] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* res = fft_smem<true>(a, b, n, W, 1, W, tw, D, dir);
  for (int t = threadIdx.x; t < n * W; t += blockDim.x) {
    const int y = t / W, q = t - y * W;
    if (q < wv) base[(int64_t)y * pc + q] = res[y * W + q];
  }
}

// ---- Z pass: forward FFT along z, multiply by the Green table g[kz][ky][kx], inverse.
// grid = (b*n+y, kx block).
__global__ void k_fft_z_green(float2* __restrict__ c, const float* __restrict__ g, FFTDesc D, int W, int pc,
                              int64_t plc) {
  extern __shared__ float2 sm[];
  const int n = D.n, nh = n / 2 + 1;
  float2* tw = sm;
  float2* a = sm + n;
  float2* b = a + W * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = D.tw[i];
  const int64_t by = blockIdx.x;  // b*n + y
  const int64_t bb = by / n;
  const int y = (int)(by - bb * n);
  const int kx0 = blockIdx.y * W;
  const int wv = min(W, nh - kx0);
  const int64_t zstride = plc;
  float2* base = c + bb * (int64_t)n * zstride + (int64_t)y * pc + kx0;
  for (int t = threadIdx.x; t < n * W; t += blockDim.x) {
    const int z = t / W, q = t - z * W;
    a[z * W + q] = (q < wv) ? base[(int64_t)z * zstride + q] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* res = fft_smem<true>(a, b, n, W, 1, W, tw, D, -1);
  const float* gb = g + (int64_t)y * nh + kx0;  // dense table, pitch nh
  for (int t = threadIdx.x; t < n * W; t += blockDim.x) {
    const int z = t / W, q = t - z * W;
    if (q < wv) {
      const float gv = gb[(int64_t)z * n * nh + q];
      float2 v = res[z * W + q];
      res[z * W + q] = make_float2(v.x * gv, v.y * gv);
    }
  }
  __syncthreads();
  float2* other = (res == a) ? b : a;
  float2* res2 = fft_smem<true>(res, other, n, W, 1, W, tw, D, +1);
  for (int t = threadIdx.x; t < n * W; t += blockDim.x) {
    const int z = t / W, q = t - z * W;
    if (q < wv) base[(int64_t)z * zstride + q] = res2[z * W + q];
  }
}

// ---- X' pass: half spectrum rows -> real rows, divided `reps` times by `norm`
// (PM1: three times by nw, pencil_fft.f90:77; PM2/PM3: once by nwork^3, kick.f90:846).
__global__ void k_fft_x_c2r(const float2* c, float* r, int64_t nrows, FFTDesc D, int rpb, float inv,
                            int pc, int pf) {
  extern __shared__ float2 sm[];
  const int n = D.n, nh = n / 2 + 1;
  float2* tw = sm;
  float2* a = sm + n;
  float2* b = a + rpb * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = D.tw[i];
  const int64_t row0 = (int64_t)blockIdx.x * rpb;
  const int nr = (int)min((int64_t)rpb, nrows - row0);
  for (int t = threadIdx.x; t < nr * n; t += blockDim.x) {
    const int rr = t / n, x = t - rr * n;
    float2 v;
    if (x < nh) {
      v = c[(row0 + rr) * pc + x];
      if (x == 0 || 2 * x == n) v.y = 0.f;
    } else {
      v = c[(row0 + rr) * pc + (n - x)];
      v.y = -v.y;
    }
    a[t] = v;
  }
  __syncthreads();
  float2* res = fft_smem<false>(a, b, n, nr, n, 1, tw, D, +1);
  for (int t = threadIdx.x; t < nr * n; t += blockDim.x) {
    const float v = __fmul_rn(res[t].x, inv);
    const int rr = t / n, x = t - rr * n;
    r[(row0 + rr) * pf + x] = v;
  }
}

}  // namespace cube
