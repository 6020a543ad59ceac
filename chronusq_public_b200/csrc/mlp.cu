// Kernels of the learned initial-density model: a small MLP trained and evaluated on the
// GPU with BF16 operands and FP32 accumulation.
//
//   k_gemm_bf16 : C[m][n] (+)= sum_k A(m,k) B(n,k), A and B BF16 with arbitrary strides
//                 (transposes are strides), FP32 accumulation in registers over 64x64
//                 tiles staged through shared memory; optional fused epilogue
//                 Z = C + bias (FP32) and Y = SiLU(Z) (BF16).
//   k_silu_bwd  : dZ = dY * SiLU'(Z)  (BF16 out, the next GEMM's operand)
//   k_colsum    : db[n] = sum_m dZ[m][n]
//   k_mse       : masked squared error, its gradient, and the loss sum
//   k_adam      : Adam step on FP32 master weights, BF16 copy for the next pass
//   k_cast_bf16 : FP32 -> BF16
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cqgpu.h"

namespace {

constexpr int TM = 64, TN = 64, TK = 16;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// 256 threads, each computes a 4x4 sub-tile of the 64x64 output tile.
__global__ void __launch_bounds__(256) k_gemm_bf16(const __nv_bfloat16 *__restrict__ A, long long sam, long long sak,
                                                   const __nv_bfloat16 *__restrict__ B, long long sbn, long long sbk,
                                                   float *__restrict__ C, long long ldc, int M, int N, int K,
                                                   const float *__restrict__ bias, __nv_bfloat16 *__restrict__ Y,
                                                   long long ldy, int act, int accumulate) {
  __shared__ float As[TK][TM + 1];
  __shared__ float Bs[TK][TN + 1];
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const int tr = tid / 16, tc = tid % 16;   // 16 x 16 threads, 4x4 outputs each
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int e = tid; e < TK * TM; e += 256) {
      const int kk = e / TM, mm = e % TM;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? __bfloat162float(A[m * sam + k * sak]) : 0.f;
    }
    for (int e = tid; e < TK * TN; e += 256) {
      const int kk = e / TN, nn = e % TN;
      const int n = n0 + nn, k = k0 + kk;
      Bs[kk][nn] = (n < N && k < K) ? __bfloat162float(B[n * sbn + k * sbk]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tr * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tc * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int m = m0 + tr * 4 + i, n = n0 + tc * 4 + j;
      if (m >= M || n >= N) continue;
      float z = acc[i][j] + (bias ? bias[n] : 0.f);
      if (accumulate) z += C[m * ldc + n];
      C[m * ldc + n] = z;
      if (Y) Y[m * ldy + n] = __float2bfloat16(act ? silu(z) : z);
    }
}

__global__ void k_silu_bwd(const float *__restrict__ dY, const float *__restrict__ Z, __nv_bfloat16 *__restrict__ dZ,
                           long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dZ[i] = __float2bfloat16(dY[i] * silu_grad(Z[i]));
}

__global__ void k_to_bf16(const float *__restrict__ x, __nv_bfloat16 *__restrict__ y, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

__global__ void k_colsum(const __nv_bfloat16 *__restrict__ dZ, int M, int N, float *__restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += __bfloat162float(dZ[(long long)m * N + n]);
  db[n] = s;
}

// loss = sum mask*(pred-target)^2 / count ; dpred = 2 mask (pred-target) / count
__global__ void k_mse(const float *__restrict__ pred, const float *__restrict__ target, const float *__restrict__ mask,
                      long long n, float inv_count, float *__restrict__ dpred, float *__restrict__ loss) {
  __shared__ float red[256];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < n) {
    const float w = mask ? mask[i] : 1.f;
    const float d = pred[i] - target[i];
    dpred[i] = 2.f * w * d * inv_count;
    l = w * d * d * inv_count;
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, long long n, float lr, float b1, float b2, float eps, float bc1,
                       float bc2, float wd, __nv_bfloat16 *__restrict__ wbf) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * w[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  const float upd = lr * (a / bc1) / (sqrtf(b / bc2) + eps);
  w[i] -= upd;
  if (wbf) wbf[i] = __float2bfloat16(w[i]);
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" {

cqg_status cqg_mlp_gemm_bf16(const void *A, long long sam, long long sak, const void *B, long long sbn, long long sbk,
                             float *C, long long ldc, int M, int N, int K, const float *bias, void *Y, long long ldy,
                             int act, int accumulate, void *stream) {
  if (!A || !B || !C || M < 0 || N < 0 || K < 0) return CQG_ERR_BAD_ARG;
  if (M == 0 || N == 0) return CQG_OK;
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  k_gemm_bf16<<<grid, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)A, sam, sak, (const __nv_bfloat16 *)B,
                                                      sbn, sbk, C, ldc, M, N, K, bias, (__nv_bfloat16 *)Y, ldy, act,
                                                      accumulate);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

cqg_status cqg_mlp_silu_bwd(const float *dY, const float *Z, void *dZ, long long n, void *stream) {
  if (n <= 0) return CQG_OK;
  k_silu_bwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(dY, Z, (__nv_bfloat16 *)dZ, n);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

cqg_status cqg_mlp_to_bf16(const float *x, void *y, long long n, void *stream) {
  if (n <= 0) return CQG_OK;
  k_to_bf16<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16 *)y, n);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

cqg_status cqg_mlp_colsum(const void *dZ, int M, int N, float *db, void *stream) {
  if (N <= 0) return CQG_OK;
  k_colsum<<<nblk(N, 128), 128, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)dZ, M, N, db);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

cqg_status cqg_mlp_mse(const float *pred, const float *target, const float *mask, long long n, float inv_count,
                       float *dpred, float *loss, void *stream) {
  if (n <= 0) return CQG_OK;
  k_mse<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(pred, target, mask, n, inv_count, dpred, loss);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

cqg_status cqg_mlp_adam(float *w, const float *g, float *m1, float *m2, long long n, float lr, float b1, float b2,
                        float eps, int step, float weight_decay, void *wbf, void *stream) {
  if (n <= 0 || step < 1) return CQG_ERR_BAD_ARG;
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_adam<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m1, m2, n, lr, b1, b2, eps, bc1, bc2, weight_decay,
                                                         (__nv_bfloat16 *)wbf);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

}  // extern "C"
