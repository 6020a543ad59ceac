// Kernels of the learned initial-density model: a small MLP trained and evaluated on the
// GPU with BF16 operands and FP32 accumulation.
//
//   k_gemm_bf16 : C[m][n] (+)= sum_k A(m,k) B(n,k), A and B BF16 with arbitrary strides
//                 (transposes are strides), on the tensor cores: mma.sync m16n8k16 BF16 x
//                 BF16 -> FP32 over 128 x 128 x 32 block tiles staged in shared memory
//                 (8 warps, 32 x 64 each); optional fused epilogue Z = C + bias (FP32) and
//                 Y = SiLU(Z) (BF16).
//   k_silu_bwd  : dZ = dY * SiLU'(Z)  (BF16 out, the next GEMM's operand)
//   k_colsum    : db[n] = sum_m dZ[m][n]
//   k_mse       : masked squared error, its gradient, and the loss sum
//   k_adam      : Adam step on FP32 master weights, BF16 copy for the next pass
//   k_cast_bf16 : FP32 -> BF16
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/cqgpu.h"

namespace {

constexpr int GM = 128, GN = 128, GK = 32, GKP = GK + 8;   // large block tile; padded smem rows

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// D += A B for one 16 x 8 x 16 tile (A row-major 16 x 16, B column-major 16 x 8, BF16
// operands, FP32 accumulators).  Fragments (g = lane / 4, t = lane % 4):
//   a[0] = A[g][2t..2t+1], a[1] = A[g+8][2t..], a[2] = A[g][2t+8..], a[3] = A[g+8][2t+8..]
//   b[0] = B[2t..2t+1][g], b[1] = B[2t+8..2t+9][g]
//   d[0..1] = D[g][2t..2t+1], d[2..3] = D[g+8][2t..2t+1]
__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Stage rows [r0, r0 + 128) x k [k0, k0 + 32) of X(r, k) = X[r * sr + k * sk] into S[row][k]
// (zero outside nrows x K).  Rows or k contiguous and 16-byte aligned: 8-element vector
// loads; anything else element by element.
template <int ROWS>
__device__ __forceinline__ void stage_tile(const __nv_bfloat16 *__restrict__ X, long long sr, long long sk, int r0,
                                           int nrows, int k0, int K, bool vec_k, bool vec_r,
                                           __nv_bfloat16 (*S)[GKP]) {
  const int tid = threadIdx.x, nth = blockDim.x;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  if (vec_k) {                 // sk == 1, sr % 8 == 0, K % 8 == 0, X 16-byte aligned
    for (int e = tid; e < ROWS * (GK / 8); e += nth) {
      const int rr = e / (GK / 8), kv = (e % (GK / 8)) * 8;
      const int r = r0 + rr, k = k0 + kv;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (r < nrows && k < K) v = *reinterpret_cast<const uint4 *>(X + (long long)r * sr + k);
      *reinterpret_cast<uint4 *>(&S[rr][kv]) = v;
    }
  } else if (vec_r) {          // sr == 1, sk % 8 == 0, nrows % 8 == 0, X 16-byte aligned
    for (int e = tid; e < GK * (ROWS / 8); e += nth) {
      const int kk = e / (ROWS / 8), rv = (e % (ROWS / 8)) * 8;
      const int r = r0 + rv, k = k0 + kk;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (r < nrows && k < K) v = *reinterpret_cast<const uint4 *>(X + r + (long long)k * sk);
      const __nv_bfloat16 *h = reinterpret_cast<const __nv_bfloat16 *>(&v);
#pragma unroll
      for (int i = 0; i < 8; ++i) S[rv + i][kk] = h[i];
    }
  } else if (sk <= sr) {       // k varies fastest across threads
    for (int e = tid; e < ROWS * GK; e += nth) {
      const int rr = e / GK, kk = e % GK;
      const int r = r0 + rr, k = k0 + kk;
      S[rr][kk] = (r < nrows && k < K) ? X[(long long)r * sr + (long long)k * sk] : zero;
    }
  } else {                     // rows vary fastest across threads
    for (int e = tid; e < ROWS * GK; e += nth) {
      const int kk = e / ROWS, rr = e % ROWS;
      const int r = r0 + rr, k = k0 + kk;
      S[rr][kk] = (r < nrows && k < K) ? X[(long long)r * sr + (long long)k * sk] : zero;
    }
  }
}

// Block tile BM x BN (BM, BN multiples of 32), warps of 32 x WN output each (WN = 64 or 32):
// (BM / 32) x (BN / WN) warps; per 16-wide k step a warp issues 2 x (WN / 8) tensor-core
// tiles.  128 x 128 with 8 warps of 32 x 64 for large problems, 64 x 64 with 4 warps of
// 32 x 32 when the large tiles would leave most of the 148 SMs idle.
template <int BM, int BN, int WN>
__global__ void __launch_bounds__((BM / 32) * (BN / WN) * 32)
    k_gemm_bf16(const __nv_bfloat16 *__restrict__ A, long long sam, long long sak, const __nv_bfloat16 *__restrict__ B,
                long long sbn, long long sbk, float *__restrict__ C, long long ldc, int M, int N, int K,
                const float *__restrict__ bias, __nv_bfloat16 *__restrict__ Y, long long ldy, int act, int accumulate,
                int kchunk) {
  constexpr int NWM = BM / 32, NJ = WN / 8;
  __shared__ __align__(16) __nv_bfloat16 As[BM][GKP];
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][GKP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp % NWM) * 32, wn = (warp / NWM) * WN;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int g = lane >> 2, t = lane & 3;
  const bool a16 = (reinterpret_cast<uintptr_t>(A) & 15) == 0, b16 = (reinterpret_cast<uintptr_t>(B) & 15) == 0;
  const bool avk = a16 && sak == 1 && sam % 8 == 0 && K % 8 == 0;
  const bool avr = a16 && !avk && sam == 1 && sak % 8 == 0 && M % 8 == 0;
  const bool bvk = b16 && sbk == 1 && sbn % 8 == 0 && K % 8 == 0;
  const bool bvr = b16 && !bvk && sbn == 1 && sbk % 8 == 0 && N % 8 == 0;
  float acc[2][NJ][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
  // split K (kchunk > 0): this block reduces k in [kb, ke) and adds its partial tile to C
  // with atomics (C zeroed by the caller); no epilogue then
  const int kb = kchunk > 0 ? blockIdx.z * kchunk : 0, ke = kchunk > 0 ? min(K, kb + kchunk) : K;
  for (int k0 = kb; k0 < ke; k0 += GK) {
    stage_tile<BM>(A, sam, sak, m0, M, k0, ke, avk, avr, As);
    stage_tile<BN>(B, sbn, sbk, n0, N, k0, ke, bvk, bvr, Bs);
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GK; ks += 16) {
      uint32_t af[2][4], bf[NJ][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + g;
        af[i][0] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t]);
        af[i][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t]);
        af[i][2] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int c = wn + j * 8 + g;
        bf[j][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][ks + 2 * t]);
        bf[j][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) mma_16816(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm + i * 16 + g + (q >> 1) * 8, n = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        if (kchunk > 0) {
          atomicAdd(C + m * ldc + n, acc[i][j][q]);
          continue;
        }
        float z = acc[i][j][q] + (bias ? bias[n] : 0.f);
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

// db[n] += sum over rows [blockIdx.y * 256, +256) of dZ[m][n]: 32 columns x 8 row groups
// per block (a warp reads 32 consecutive columns of one row), partial sums reduced in shared
// memory, one atomic per column and block (db zeroed by the caller).
__global__ void __launch_bounds__(256) k_colsum(const __nv_bfloat16 *__restrict__ dZ, int M, int N,
                                                float *__restrict__ db) {
  __shared__ float part[8][33];
  const int c = threadIdx.x & 31, rg = threadIdx.x >> 5;
  const int n = blockIdx.x * 32 + c;
  const int m0 = blockIdx.y * 256, m1 = min(M, m0 + 256);
  float s = 0.f;
  if (n < N)
    for (int m = m0 + rg; m < m1; m += 8) s += __bfloat162float(dZ[(long long)m * N + n]);
  part[rg][c] = s;
  __syncthreads();
  if (rg == 0 && n < N) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += part[k][c];
    atomicAdd(db + n, t);
  }
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

// The same step with the learning rate and the two bias corrections read from device memory
// (hyper = {lr, 1 - b1^step, 1 - b2^step}), so that a captured training step can be replayed
// with a schedule that changes from step to step.
__global__ void k_adam_dev(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                           float *__restrict__ m2, long long n, const float *__restrict__ hyper, float b1, float b2,
                           float eps, float wd, __nv_bfloat16 *__restrict__ wbf) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float lr = hyper[0], bc1 = hyper[1], bc2 = hyper[2];
  const float gi = g[i] + wd * w[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
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
  const long long big_blocks = (long long)((N + GN - 1) / GN) * ((M + GM - 1) / GM);
  cudaStream_t st = (cudaStream_t)stream;
  const __nv_bfloat16 *a = (const __nv_bfloat16 *)A, *b = (const __nv_bfloat16 *)B;
  if (big_blocks >= 296) {   // two waves of 148 SMs or more: large tiles
    if ((M + GM - 1) / GM > 65535) return CQG_ERR_BAD_ARG;   // grid.y limit
    dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    k_gemm_bf16<GM, GN, 64><<<grid, 256, 0, st>>>(a, sam, sak, b, sbn, sbk, C, ldc, M, N, K, bias,
                                                  (__nv_bfloat16 *)Y, ldy, act, accumulate, 0);
  } else {
    if ((M + 63) / 64 > 65535) return CQG_ERR_BAD_ARG;
    const long long tiles = (long long)((N + 63) / 64) * ((M + 63) / 64);
    // few output tiles and a long reduction (weight gradients: K = batch rows): split K over
    // blockIdx.z so that about two waves of CTAs run, partial tiles added with atomics
    int splits = 1;
    if (!bias && !Y && tiles < 148 && K >= 4 * GK) {
      splits = (int)std::min<long long>((296 + tiles - 1) / tiles, K / (2 * GK));
      splits = std::max(1, std::min(splits, 64));
    }
    const int kchunk = splits > 1 ? ((K + splits - 1) / splits + GK - 1) / GK * GK : 0;
    if (kchunk > 0) {
      splits = (K + kchunk - 1) / kchunk;
      if (!accumulate) {
        if (cudaMemset2DAsync(C, ldc * sizeof(float), 0, N * sizeof(float), M, st) != cudaSuccess) return CQG_ERR_CUDA;
      }
    }
    dim3 grid((N + 63) / 64, (M + 63) / 64, splits);
    k_gemm_bf16<64, 64, 32><<<grid, 128, 0, st>>>(a, sam, sak, b, sbn, sbk, C, ldc, M, N, K, bias,
                                                  (__nv_bfloat16 *)Y, ldy, act, accumulate, kchunk);
  }
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
  if (cudaMemsetAsync(db, 0, (size_t)N * sizeof(float), (cudaStream_t)stream) != cudaSuccess) return CQG_ERR_CUDA;
  if (M <= 0) return CQG_OK;
  if ((M + 255) / 256 > 65535) return CQG_ERR_BAD_ARG;
  dim3 grid((N + 31) / 32, (M + 255) / 256);
  k_colsum<<<grid, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)dZ, M, N, db);
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

cqg_status cqg_mlp_adam_dev(float *w, const float *g, float *m1, float *m2, long long n, const float *hyper,
                            float b1, float b2, float eps, float weight_decay, void *wbf, void *stream) {
  if (n <= 0 || !hyper) return CQG_ERR_BAD_ARG;
  k_adam_dev<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m1, m2, n, hyper, b1, b2, eps, weight_decay,
                                                             (__nv_bfloat16 *)wbf);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

}  // extern "C"
