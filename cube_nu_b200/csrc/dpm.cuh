// Differentiable particle-mesh step and its hand-written adjoint (the PyTorch binding
// cube_nu_b200/adjoint.py wraps these behind torch.autograd.Function).  Included by
// cube_gpu.cu after kernels.cuh.
//
// The forward is one PM level on a periodic n^3 mesh in fine-cell units, with the
// reference's PM pieces: TSC mass assignment with the cell-centred convention of
// particle_mesh.f90:56-62 (cells floor(x)-1 .. floor(x)+1, l = x - floor(x)), the Green
// table of Green/Green.f90 applied between a forward and an inverse FFT, the 4-point
// gradient of the potential (particle_mesh.f90:224-247) and TSC interpolation of the
// force, in the KDK order of main.f90 (drift, then kick with dv = F * a_mid * dt/(6 pi)).
// Positions are real (not ZIPX codes), so the step is differentiable.
//
// Adjoints, for a cotangent u_i of the particle forces F_i = sum_c W(x_i - c) Fm(c),
// Fm = grad_h phi, phi = Gconv(rho), rho(c) = m sum_j W(x_j - c):
//   d(u.F)/dx_k = sum_c dW(x_k - c) (u_k . Fm(c))            (interpolation weights)
//               + m sum_c dW(x_k - c) psi(c)                 (mass assignment weights)
//   psi = Gconv(grad_h^T lamF),  lamF(c) = sum_i W(x_i - c) u_i
// Gconv is symmetric (a real Green table), grad_h^T = -grad_h (antisymmetric stencil).
#pragma once
#include "kernels.cuh"

namespace cube {

// 1-D TSC weights and their derivatives at x (fine units): cells fl-1, fl, fl+1.
__device__ __forceinline__ int dpm_w(float x, float w[3], float dw[3]) {
  const float fl = floorf(x);
  const float l = x - fl;
  const float a = 1.f - l;
  w[0] = 0.5f * a * a;
  w[2] = 0.5f * l * l;
  w[1] = 1.f - w[0] - w[2];
  dw[0] = -a;
  dw[2] = l;
  dw[1] = a - l;
  return (int)fl;
}

__device__ __forceinline__ int dpm_wrap(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// rho += m * W, into a mesh with row pitch pr and plane pitch pl (floats).
__global__ void k_dpm_deposit(int n, int64_t np, const float* __restrict__ x, float m, float* __restrict__ rho, int pr,
                              int64_t pl) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float w[3][3], dw[3];
  int f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) f[d] = dpm_w(x[3 * i + d], w[d], dw);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t z = (int64_t)dpm_wrap(f[2] - 1 + c, n) * pl;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int64_t y = (int64_t)dpm_wrap(f[1] - 1 + b, n) * pr;
#pragma unroll
      for (int a = 0; a < 3; ++a) atomicAdd(&rho[z + y + dpm_wrap(f[0] - 1 + a, n)], m * w[0][a] * w[1][b] * w[2][c]);
    }
  }
}

// F_i = sum_c W Fm(c) (Fm: float4 per cell, dense, x fastest); then the KDK kick
// v += K F and, with D != 0, the next drift is not applied here.
__global__ void k_dpm_kick(int n, int64_t np, const float* __restrict__ x, const float4* __restrict__ fm, float K,
                           float* __restrict__ v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float w[3][3], dw[3];
  int f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) f[d] = dpm_w(x[3 * i + d], w[d], dw);
  float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t z = (int64_t)dpm_wrap(f[2] - 1 + c, n) * n * n;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int64_t y = (int64_t)dpm_wrap(f[1] - 1 + b, n) * n;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float4 F = __ldg(&fm[z + y + dpm_wrap(f[0] - 1 + a, n)]);
        const float ww = w[0][a] * w[1][b] * w[2][c];
        s0 += ww * F.x;
        s1 += ww * F.y;
        s2 += ww * F.z;
      }
    }
  }
  v[3 * i] += K * s0;
  v[3 * i + 1] += K * s1;
  v[3 * i + 2] += K * s2;
}

// x += D v, wrapped into [0, n).
__global__ void k_dpm_drift(int n, int64_t np3, float* __restrict__ x, const float* __restrict__ v, float D) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np3) return;
  float y = x[i] + D * v[i];
  const float fn = (float)n;
  y -= fn * floorf(y / fn);
  if (y >= fn) y -= fn;  // rounding of y / fn just below an integer
  x[i] = y;
}

// lamF(c) += sum_i W(x_i - c) u_i (float4 mesh, dense, x fastest; .w unused).
__global__ void k_dpm_deposit_vec(int n, int64_t np, const float* __restrict__ x, const float* __restrict__ u,
                                  float4* __restrict__ lam) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float w[3][3], dw[3];
  int f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) f[d] = dpm_w(x[3 * i + d], w[d], dw);
  const float u0 = u[3 * i], u1 = u[3 * i + 1], u2 = u[3 * i + 2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t z = (int64_t)dpm_wrap(f[2] - 1 + c, n) * n * n;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int64_t y = (int64_t)dpm_wrap(f[1] - 1 + b, n) * n;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float* L = reinterpret_cast<float*>(&lam[z + y + dpm_wrap(f[0] - 1 + a, n)]);
        const float ww = w[0][a] * w[1][b] * w[2][c];
        atomicAdd(L, ww * u0);
        atomicAdd(L + 1, ww * u1);
        atomicAdd(L + 2, ww * u2);
      }
    }
  }
}

// s(c) = (grad_h^T lamF)(c) = sum_d sum_o w_o lamF_d(c - o e_d), o in {-2,-1,1,2}, the
// transpose of the 4-point gradient; written into a mesh with row pitch pr, plane pl.
__global__ void k_dpm_grad_t(int n, const float4* __restrict__ lam, float* __restrict__ s, int pr, int64_t pl) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n3 = (int64_t)n * n * n;
  if (i >= n3) return;
  const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
  const float w[4] = {(CUBE_W_ALPHA - 1.f) / 4.f, -CUBE_W_ALPHA / 2.f, CUBE_W_ALPHA / 2.f, (1.f - CUBE_W_ALPHA) / 4.f};
  const int o[4] = {-2, -1, 1, 2};
  auto L = [&](int a, int b, int c) { return __ldg(&lam[((int64_t)c * n + b) * n + a]); };
  float t = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    t += w[k] * L(dpm_wrap(x - o[k], n), y, z).x;
    t += w[k] * L(x, dpm_wrap(y - o[k], n), z).y;
    t += w[k] * L(x, y, dpm_wrap(z - o[k], n)).z;
  }
  s[(int64_t)z * pl + (int64_t)y * pr + x] = t;
}

// gx_k += sum_c dW(x_k - c) (u_k . Fm(c) + m psi(c)) over the 27 TSC cells; u or psi may be
// null (density adjoint: u = null, psi = lam with m the mass).
__global__ void k_dpm_grad_gather(int n, int64_t np, const float* __restrict__ x, const float* __restrict__ u,
                                  const float4* __restrict__ fm, const float* __restrict__ psi, int pr, int64_t pl,
                                  float m, float* __restrict__ gx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float w[3][3], dw[3][3];
  int f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) f[d] = dpm_w(x[3 * i + d], w[d], dw[d]);
  const float u0 = u ? u[3 * i] : 0.f, u1 = u ? u[3 * i + 1] : 0.f, u2 = u ? u[3 * i + 2] : 0.f;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int zz = dpm_wrap(f[2] - 1 + c, n);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int yy = dpm_wrap(f[1] - 1 + b, n);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int xx = dpm_wrap(f[0] - 1 + a, n);
        float val = 0.f;
        if (u) {
          const float4 F = __ldg(&fm[((int64_t)zz * n + yy) * n + xx]);
          val = u0 * F.x + u1 * F.y + u2 * F.z;
        }
        if (psi) val += m * __ldg(&psi[(int64_t)zz * pl + (int64_t)yy * pr + xx]);
        g0 += dw[0][a] * w[1][b] * w[2][c] * val;
        g1 += w[0][a] * dw[1][b] * w[2][c] * val;
        g2 += w[0][a] * w[1][b] * dw[2][c] * val;
      }
    }
  }
  gx[3 * i] += g0;
  gx[3 * i + 1] += g1;
  gx[3 * i + 2] += g2;
}

// Copy a pitched mesh (row pr, plane pl) into a dense n^3 array, or back.
__global__ void k_dpm_copy(int n, const float* __restrict__ src, int spr, int64_t spl, float* __restrict__ dst, int dpr,
                           int64_t dpl) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n3 = (int64_t)n * n * n;
  if (i >= n3) return;
  const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
  dst[(int64_t)z * dpl + (int64_t)y * dpr + x] = src[(int64_t)z * spl + (int64_t)y * spr + x];
}

}  // namespace cube
