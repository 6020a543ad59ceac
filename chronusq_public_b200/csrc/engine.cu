// cqgpu engine: direct-SCF two-electron contraction G[X] = J - K on sm_100a.
//
// Data flow of one contraction (the reference loop it replaces is
// include/aointegrals/aointegrals_contract.h:24-194):
//   1. k_blocknorm   : M(s1,s2) = max_i max|X_i block|  (computeShBlkNorm, basisset.h:495-509),
//                      plus non-finite / asymmetry flags.
//   2. k_quartet_count / scan / k_quartet_fill : the unique shell quartets that pass the
//                      density-weighted Schwarz screen (contract.h:112-131), grouped by
//                      angular-momentum class, bra-major, as (bra pair, ket pair) indices.
//   3. k_eri_jk<class> : one thread per quartet: McMurchie-Davidson ERIs (generated code)
//                      and the J/K digest of contract.h:145-171 (half of the updates; the
//                      other half is the transpose) with FP64 atomics into Gh.
//   4. k_finalize    : AX += 0.5 (Gh + Gh^T)   (the 0.5*scale reduction of contract.h:189-193;
//                      the scales are folded into the digest).
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/cqgpu.h"
#include "eri_common.cuh"
#include "_gen/eri_classes.cuh"

#define CQG_MAXL 2
#define CQG_NPC ((CQG_MAXL + 1) * (CQG_MAXL + 2) / 2)       // pair classes
#define CQG_NQC (CQG_NPC * (CQG_NPC + 1) / 2)                // quartet classes
#define CQG_MAXG 4

static_assert(CQG_NQC <= 55, "class table");

// ------------------------------------------------------------------ class tables ---
static const int kPairClass[10][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2},
                                      {3, 0}, {3, 1}, {3, 2}, {3, 3}};
static inline int pair_class_of(int la, int lb) {  // la >= lb
  return la * (la + 1) / 2 + lb;
}
static inline int nfun(int l) { return l > 1 ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nfun_c(int l) { return l > 1 ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int ncart_c(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nherm_c(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }

// quartet class k <-> (bra pair class i, ket pair class j), i >= j, k = i(i+1)/2 + j
static inline void qclass_split(int k, int &i, int &j) {
  i = 0;
  while ((i + 1) * (i + 2) / 2 <= k) ++i;
  j = k - i * (i + 1) / 2;
}

static const char *kLetters = "spdfg";
static char g_class_names[55][16];
static bool g_names_init = false;

// MD-v1 model FLOPs per primitive quartet and per quartet digest, for class (la lb|lc ld).
static double md_v1_prim_flops(int la, int lb, int lc, int ld) {
  int p = la + lb, q = lc + ld, L = p + q;
  double c4 = (double)(L + 4) * (L + 3) * (L + 2) * (L + 1) / 24.0;
  return 30.0 + 3.0 * L + 2.0 * c4 + 2.0 * ncart_c(lc) * ncart_c(ld) * nherm_c(p) * nherm_c(q) +
         2.0 * ncart_c(la) * ncart_c(lb) * ncart_c(lc) * ncart_c(ld) * nherm_c(p);
}
static double md_v1_digest_flops(int la, int lb, int lc, int ld) {
  return 24.0 * nfun(la) * nfun(lb) * nfun(lc) * nfun(ld);
}

// ------------------------------------------------------------------ device data ---
struct Shells {
  const double3 *center;
  const int *bf;
};
struct Pairs {
  const int2 *sh;       // (shell a, shell b), internal orientation L_a >= L_b
  const double *Q;      // Schwarz bound
  const int *poff;      // first primitive pair
  const int *np;        // number of primitive pairs
  const PrimPair *prim;
};
struct DigestGroups {
  const double *X[CQG_MAXG];
  double *G[CQG_MAXG];
  double sJ[CQG_MAXG];
  double sK[CQG_MAXG];
  int ng;
  int ldx;
  int n;
};

// ------------------------------------------------------------------ kernels ---
// Schwarz: Q(ab) = sqrt(max_ij |(ij|ij)|) for pairs [beg, end) of one class.
template <int LA, int LB>
__global__ void __launch_bounds__(128) k_schwarz(Pairs P, Shells S, const double *__restrict__ boys,
                                                 int beg, int end, double *__restrict__ Qout) {
  int i = beg + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= end) return;
  constexpr int NA = nfun_c(LA), NB = nfun_c(LB), NAB = NA * NB;
  int2 s = P.sh[i];
  double3 A = S.center[s.x], B = S.center[s.y];
  double out[NAB * NAB];
  const PrimPair *pp = P.prim + P.poff[i];
  EriClass<LA, LB, LA, LB>::template run<double>(pp, P.np[i], pp, P.np[i], A, B, A, B, boys, out);
  double mx = 0.0;
#pragma unroll
  for (int ij = 0; ij < NAB; ++ij) mx = fmax(mx, fabs(out[ij * NAB + ij]));
  Qout[i] = sqrt(mx);
}

// Block norms M(s1,s2) = max over matrices of max|X_i(block)|, and input checks.
struct XList {
  const double *X[8];
  int n;
};
__global__ void k_blocknorm(XList xl, int ldx, int nsh, const int *__restrict__ bf,
                            const int *__restrict__ sz, double *__restrict__ M,
                            int *__restrict__ flags, double sym_tol) {
  int s1 = blockIdx.x * blockDim.x + threadIdx.x;
  int s2 = blockIdx.y;
  if (s1 >= nsh) return;
  int r0 = bf[s1], c0 = bf[s2], nr = sz[s1], nc = sz[s2];
  double mx = 0.0;
  int bad = 0, asym = 0;
  for (int m = 0; m < xl.n; ++m) {
    const double *X = xl.X[m];
    for (int c = 0; c < nc; ++c)
      for (int r = 0; r < nr; ++r) {
        double v = X[(size_t)(r0 + r) + (size_t)(c0 + c) * ldx];
        double t = X[(size_t)(c0 + c) + (size_t)(r0 + r) * ldx];
        if (!isfinite(v)) bad = 1;
        double av = fabs(v);
        mx = fmax(mx, av);
        if (fabs(v - t) > sym_tol * fmax(1.0, av)) asym = 1;
      }
  }
  M[(size_t)s1 + (size_t)s2 * nsh] = mx;
  if (bad) atomicOr(flags + 0, 1);
  if (asym) atomicOr(flags + 1, 1);
}

__global__ void k_maxreduce(const double *__restrict__ M, long long n, double *__restrict__ out) {
  __shared__ double sm[32];
  double mx = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    mx = fmax(mx, M[i]);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    mx = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (threadIdx.x == 0) {
      // non-negative doubles order like their bit patterns
      atomicMax((unsigned long long *)out, (unsigned long long)__double_as_longlong(mx));
    }
  }
}

// One screening task = (class block, bra pair).  Blocks are listed in task order.
struct BlockTable {
  int nblk;
  int task_beg[CQG_NQC + 1];   // first task of each block
  int bra_beg[CQG_NQC];        // first bra pair (global index) of the block
  int ket_beg[CQG_NQC];        // first ket pair (global index) of the block
  int ket_n[CQG_NQC];          // number of ket pairs of the block's ket class
  int diag[CQG_NQC];           // bra class == ket class
};

__device__ __forceinline__ int find_block(const BlockTable &bt, int task) {
  int b = 0;
  while (b + 1 < bt.nblk && bt.task_beg[b + 1] <= task) ++b;
  return b;
}

// number of ket pairs (from the start of the Q-descending ket list) that can pass
__device__ __forceinline__ int coarse_range(const double *__restrict__ Q, int kb, int kn, double cut) {
  // first index with Q < cut
  int lo = 0, hi = kn;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (Q[kb + mid] >= cut) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool exact_pass(const double *__restrict__ M, int nsh, int2 ab, int2 cd,
                                           double qab, double qcd, double thresh) {
  const int s1 = ab.x, s2 = ab.y, s3 = cd.x, s4 = cd.y;
  double m = M[s1 + (size_t)s4 * nsh];
  m = fmax(m, M[s2 + (size_t)s4 * nsh]);
  m = fmax(m, M[s3 + (size_t)s4 * nsh]);
  m = fmax(m, M[s1 + (size_t)s3 * nsh]);
  m = fmax(m, M[s2 + (size_t)s3 * nsh]);
  m = fmax(m, M[s1 + (size_t)s2 * nsh]);
  return m * qab * qcd >= thresh;
}

// Count (FILL=false) or write (FILL=true) the passing quartets of each task.  One warp
// per task; ket pairs scanned in ascending order, survivors compacted with a ballot so
// the list is deterministic.
template <bool FILL>
__global__ void __launch_bounds__(256) k_quartets(BlockTable bt, int ntask, Pairs P, const double *__restrict__ M,
                                                  int nsh, const double *__restrict__ Mmax, double thresh,
                                                  long long *__restrict__ cnt, const long long *__restrict__ off,
                                                  uint2 *__restrict__ qlist) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ntask) return;
  int blk = find_block(bt, warp);
  int bra = bt.bra_beg[blk] + (warp - bt.task_beg[blk]);
  double qb = P.Q[bra];
  double mm = *Mmax;
  int kn = bt.ket_n[blk];
  int nk = 0;
  if (qb * mm > 0.0) {
    double cut = thresh / (qb * mm) * (1.0 - 1e-12);
    nk = coarse_range(P.Q, bt.ket_beg[blk], kn, cut);
  }
  if (bt.diag[blk]) nk = min(nk, bra - bt.bra_beg[blk] + 1);
  int2 ab = P.sh[bra];
  long long base = FILL ? off[warp] : 0;
  long long c = 0;
  for (int k0 = 0; k0 < nk; k0 += 32) {
    int k = k0 + lane;
    bool pass = false;
    int ket = bt.ket_beg[blk] + k;
    if (k < nk) pass = exact_pass(M, nsh, ab, P.sh[ket], qb, P.Q[ket], thresh);
    unsigned bal = __ballot_sync(0xffffffffu, pass);
    if (FILL && pass) {
      int pos = __popc(bal & ((1u << lane) - 1u));
      qlist[base + c + pos] = make_uint2((unsigned)bra, (unsigned)ket);
    }
    c += __popc(bal);
  }
  if (!FILL && lane == 0) cnt[warp] = c;
}

// block ranges [beg, end) of the quartet list from the per-task counts and offsets
__global__ void k_block_ranges(BlockTable bt, const long long *__restrict__ cnt, const long long *__restrict__ off,
                               long long *__restrict__ range) {
  int b = threadIdx.x;
  if (b >= bt.nblk) return;
  int t0 = bt.task_beg[b], t1 = bt.task_beg[b + 1];
  long long beg = 0, end = 0;
  if (t1 > t0) {
    beg = off[t0];
    end = off[t1 - 1] + cnt[t1 - 1];
  } else if (t0 > 0) {
    beg = end = off[t0 - 1] + cnt[t0 - 1];
  }
  range[2 * b] = beg;
  range[2 * b + 1] = end;
}

template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void digest(const double *v, double deg, int a0, int b0, int c0, int d0,
                                       const DigestGroups &dg) {
  const size_t ld = dg.ldx, n = dg.n;
  for (int g = 0; g < dg.ng; ++g) {
    const double *__restrict__ X = dg.X[g];
    double *G = dg.G[g];
    const double sJ = dg.sJ[g] * deg;
    const double sK = 0.5 * dg.sK[g] * deg;
    if (sJ != 0.0) {
      double xdc[NC * ND], xba[NA * NB];
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) xdc[c * ND + d] = __ldg(X + (d0 + d) + (c0 + c) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) xba[a * NB + b] = __ldg(X + (b0 + b) + (a0 + a) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          double s = 0.0;
#pragma unroll
          for (int cd = 0; cd < NC * ND; ++cd) s += xdc[cd] * v[(a * NB + b) * NC * ND + cd];
          atomicAdd(G + (a0 + a) + (b0 + b) * n, sJ * s);
        }
#pragma unroll
      for (int cd = 0; cd < NC * ND; ++cd) {
        double s = 0.0;
#pragma unroll
        for (int ab = 0; ab < NA * NB; ++ab) s += xba[ab] * v[ab * NC * ND + cd];
        atomicAdd(G + (c0 + cd / ND) + (d0 + cd % ND) * n, sJ * s);
      }
    }
    if (sK != 0.0) {
      // G(a,c) += X(b,d) v ; G(b,d) += X(a,c) v ; G(a,d) += X(b,c) v ; G(b,c) += X(a,d) v
      double xbd[NB * ND], xac[NA * NC], xbc[NB * NC], xad[NA * ND];
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int d = 0; d < ND; ++d) xbd[b * ND + d] = __ldg(X + (b0 + b) + (d0 + d) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) xac[a * NC + c] = __ldg(X + (a0 + a) + (c0 + c) * ld);
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) xbc[b * NC + c] = __ldg(X + (b0 + b) + (c0 + c) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int d = 0; d < ND; ++d) xad[a * ND + d] = __ldg(X + (a0 + a) + (d0 + d) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int d = 0; d < ND; ++d) s += xbd[b * ND + d] * v[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (a0 + a) + (c0 + c) * n, sK * s);
        }
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          double s = 0.0;
#pragma unroll
          for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int c = 0; c < NC; ++c) s += xac[a * NC + c] * v[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (b0 + b) + (d0 + d) * n, sK * s);
        }
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int c = 0; c < NC; ++c) s += xbc[b * NC + c] * v[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (a0 + a) + (d0 + d) * n, sK * s);
        }
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s = 0.0;
#pragma unroll
          for (int a = 0; a < NA; ++a)
#pragma unroll
            for (int d = 0; d < ND; ++d) s += xad[a * ND + d] * v[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (b0 + b) + (c0 + c) * n, sK * s);
        }
    }
  }
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) k_eri_jk(const uint2 *__restrict__ ql, const long long *__restrict__ range,
                                                int blk, Pairs P, Shells S, const double *__restrict__ boys,
                                                DigestGroups dg) {
  const long long beg = range[2 * blk], end = range[2 * blk + 1];
  const long long i = beg + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= end) return;
  constexpr int NA = nfun_c(LA), NB = nfun_c(LB), NC = nfun_c(LC), ND = nfun_c(LD);
  const uint2 e = ql[i];
  const int2 ab = P.sh[e.x], cd = P.sh[e.y];
  const double3 A = S.center[ab.x], B = S.center[ab.y], C = S.center[cd.x], D = S.center[cd.y];
  double v[NA * NB * NC * ND];
  EriClass<LA, LB, LC, LD>::template run<double>(P.prim + P.poff[e.x], P.np[e.x], P.prim + P.poff[e.y],
                                                 P.np[e.y], A, B, C, D, boys, v);
  const double deg = (ab.x == ab.y ? 1.0 : 2.0) * (cd.x == cd.y ? 1.0 : 2.0) * (e.x == e.y ? 1.0 : 2.0);
  digest<NA, NB, NC, ND>(v, deg, S.bf[ab.x], S.bf[ab.y], S.bf[cd.x], S.bf[cd.y], dg);
}

// AX += 0.5 (Gh + Gh^T)
__global__ void k_finalize(const double *__restrict__ Gh, int n, double *__restrict__ AX, int ldax) {
  __shared__ double tile[32][33];
  int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int k = ty; k < 32; k += 8) {
    int r = bx + tx, c = by + k;   // load Gh(c', r') transposed tile: Gh(by+k, bx+tx)?
    (void)r; (void)c;
    int rr = by + tx, cc = bx + k;
    tile[k][tx] = (rr < n && cc < n) ? Gh[(size_t)rr + (size_t)cc * n] : 0.0;  // tile[k][tx] = Gh(by+tx, bx+k)
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    int r = bx + tx, c = by + k;
    if (r < n && c < n) {
      double g = Gh[(size_t)r + (size_t)c * n];
      double gt = tile[tx][k];  // Gh(by+k, bx+tx) = Gh(c, r)
      AX[(size_t)r + (size_t)c * ldax] += 0.5 * (g + gt);
    }
  }
}

// FMA throughput probe (roofline denominator): independent dependent-FMA chains.
template <typename T>
__global__ void k_fma_probe(T *out, int iters, T seed) {
  T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const T m = T(0.999999), c = T(1e-7);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = a0 * m + c; a1 = a1 * m + c; a2 = a2 * m + c; a3 = a3 * m + c;
      a4 = a4 * m + c; a5 = a5 * m + c; a6 = a6 * m + c; a7 = a7 * m + c;
    }
  }
  T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == T(-12345.0)) out[0] = s;
}

// ------------------------------------------------------------------ host side ---
#define CUCHK(call)                                                                \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(_e);               \
      return CQG_ERR_CUDA;                                                         \
    }                                                                              \
  } while (0)

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaError_t reserve(size_t m) {
    if (m <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    size_t want = std::max<size_t>(m, 1);
    cudaError_t e = cudaMalloc(&p, want * sizeof(T));
    if (e == cudaSuccess) n = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct cqg_ctx {
  int device = 0;
  std::string err;
  double thresh = 1e-14;
  int policy = CQG_PREC_FP64;
  double fp32_cutoff = 0.0;
  int timing = 0;
  // basis
  int nshell = 0, nbf = 0, maxl = 0;
  std::vector<int> hL, hbf, hsz, hnprim, hpoff;
  std::vector<double> halpha, hcoef, hcent;
  std::vector<double> Qmat;  // nshell x nshell
  // pairs, by class
  int pc_beg[CQG_NPC + 1] = {0};
  std::vector<int2> pair_sh;
  std::vector<double> pair_Q;
  DevBuf<double3> d_center;
  DevBuf<int> d_bf, d_sz;
  DevBuf<int2> d_pair_sh;
  DevBuf<double> d_pair_Q;
  DevBuf<int> d_pair_poff, d_pair_np;
  DevBuf<PrimPair> d_prim;
  DevBuf<double> d_boys;
  long long prim_pairs_total = 0;
  std::vector<int> pair_np_host;
  // per-call scratch
  DevBuf<double> d_M, d_Mmax;
  DevBuf<int> d_flags;
  DevBuf<long long> d_cnt, d_off, d_range;
  DevBuf<unsigned char> d_scan_tmp;
  DevBuf<uint2> d_qlist;
  DevBuf<double> d_G, d_X, d_AX;
  BlockTable bt;
  int ntask = 0;
  cudaEvent_t ev[4 + 2 * 55];
  bool events = false;
  cqg_stats stats;
};

static double host_boys_row(int nmax, long double T, double *F) {
  long double term = 1.0L / (2 * nmax + 1), sum = term;
  for (int k = 1; k < 2000; k++) {
    term *= 2.0L * T / (2 * nmax + 2 * k + 1);
    sum += term;
    if (term < sum * 1e-22L) break;
  }
  long double ex = expl(-T);
  long double f = ex * sum;
  F[nmax] = (double)f;
  for (int m = nmax - 1; m >= 0; m--) {
    f = (2.0L * T * f + ex) / (2 * m + 1);
    F[m] = (double)f;
  }
  return 0;
}

template <int LA, int LB>
static cudaError_t launch_schwarz(cqg_ctx *ctx, Pairs P, Shells S, int beg, int end, double *Q) {
  int n = end - beg;
  if (n <= 0) return cudaSuccess;
  k_schwarz<LA, LB><<<(n + 127) / 128, 128>>>(P, S, ctx->d_boys.p, beg, end, Q);
  return cudaGetLastError();
}

static Pairs make_pairs(cqg_ctx *ctx) {
  Pairs P;
  P.sh = ctx->d_pair_sh.p;
  P.Q = ctx->d_pair_Q.p;
  P.poff = ctx->d_pair_poff.p;
  P.np = ctx->d_pair_np.p;
  P.prim = ctx->d_prim.p;
  return P;
}
static Shells make_shells(cqg_ctx *ctx) {
  Shells S;
  S.center = ctx->d_center.p;
  S.bf = ctx->d_bf.p;
  return S;
}

// build primitive-pair data for the current pair ordering; prim_thresh = 0 keeps all
static cqg_status upload_pairs(cqg_ctx *ctx, double prim_thresh) {
  size_t np = ctx->pair_sh.size();
  std::vector<int> poff(np), npr(np);
  std::vector<PrimPair> prim;
  prim.reserve(np * 4);
  const double pi = 3.14159265358979323846;
  for (size_t i = 0; i < np; ++i) {
    int a = ctx->pair_sh[i].x, b = ctx->pair_sh[i].y;
    const double *A = &ctx->hcent[3 * a], *B = &ctx->hcent[3 * b];
    double AB2 = 0, ABn;
    for (int x = 0; x < 3; ++x) AB2 += (A[x] - B[x]) * (A[x] - B[x]);
    ABn = std::sqrt(AB2);
    poff[i] = (int)prim.size();
    for (int ia = 0; ia < ctx->hnprim[a]; ++ia)
      for (int ib = 0; ib < ctx->hnprim[b]; ++ib) {
        double al = ctx->halpha[ctx->hpoff[a] + ia], be = ctx->halpha[ctx->hpoff[b] + ib];
        double ca = ctx->hcoef[ctx->hpoff[a] + ia], cb = ctx->hcoef[ctx->hpoff[b] + ib];
        double p = al + be;
        double K = ca * cb * std::exp(-al * be / p * AB2);
        if (prim_thresh > 0) {
          // s-type sqrt((ij|ij)) estimate with a polynomial allowance for higher L
          double bound = std::fabs(K) * std::sqrt(2.0 * std::pow(pi, 2.5)) / (p * std::pow(2.0 * p, 0.25)) *
                         std::pow(1.0 + ABn, ctx->hL[a] + ctx->hL[b]);
          if (bound < prim_thresh) continue;
        }
        PrimPair pp;
        pp.p = p;
        pp.K = K;
        pp.Px = (al * A[0] + be * B[0]) / p;
        pp.Py = (al * A[1] + be * B[1]) / p;
        pp.Pz = (al * A[2] + be * B[2]) / p;
        pp.pad = 0;
        prim.push_back(pp);
      }
    npr[i] = (int)prim.size() - poff[i];
  }
  ctx->prim_pairs_total = (long long)prim.size();
  ctx->pair_np_host = npr;
  if (ctx->d_pair_sh.reserve(np) || ctx->d_pair_Q.reserve(np) || ctx->d_pair_poff.reserve(np) ||
      ctx->d_pair_np.reserve(np) || ctx->d_prim.reserve(prim.size())) {
    ctx->err = "device allocation for pair data failed";
    return CQG_ERR_OOM;
  }
  CUCHK(cudaMemcpy(ctx->d_pair_sh.p, ctx->pair_sh.data(), np * sizeof(int2), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_Q.p, ctx->pair_Q.data(), np * sizeof(double), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_poff.p, poff.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_np.p, npr.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  if (!prim.empty())
    CUCHK(cudaMemcpy(ctx->d_prim.p, prim.data(), prim.size() * sizeof(PrimPair), cudaMemcpyHostToDevice));
  return CQG_OK;
}

typedef cudaError_t (*eri_launcher)(cqg_ctx *, int blk, long long n, cudaStream_t st, const DigestGroups &dg);

template <int LA, int LB, int LC, int LD>
static cudaError_t launch_eri(cqg_ctx *ctx, int blk, long long n, cudaStream_t st, const DigestGroups &dg) {
  if (n <= 0) return cudaSuccess;
  long long nb = (n + 127) / 128;
  k_eri_jk<LA, LB, LC, LD><<<(unsigned)nb, 128, 0, st>>>(ctx->d_qlist.p, ctx->d_range.p, blk, make_pairs(ctx),
                                                         make_shells(ctx), ctx->d_boys.p, dg);
  return cudaGetLastError();
}

#define QC(a, b, c, d) &launch_eri<a, b, c, d>
static const eri_launcher kEriLaunch[CQG_NQC] = {
    QC(0, 0, 0, 0),
    QC(1, 0, 0, 0), QC(1, 0, 1, 0),
    QC(1, 1, 0, 0), QC(1, 1, 1, 0), QC(1, 1, 1, 1),
    QC(2, 0, 0, 0), QC(2, 0, 1, 0), QC(2, 0, 1, 1), QC(2, 0, 2, 0),
    QC(2, 1, 0, 0), QC(2, 1, 1, 0), QC(2, 1, 1, 1), QC(2, 1, 2, 0), QC(2, 1, 2, 1),
    QC(2, 2, 0, 0), QC(2, 2, 1, 0), QC(2, 2, 1, 1), QC(2, 2, 2, 0), QC(2, 2, 2, 1), QC(2, 2, 2, 2),
};
#undef QC

extern "C" {

const char *cqg_version(void) { return "cqgpu 0.1 (sm_100a, MD FP64)"; }

const char *cqg_status_string(cqg_status s) {
  switch (s) {
    case CQG_OK: return "ok";
    case CQG_ERR_BAD_ARG: return "bad argument";
    case CQG_ERR_OOM: return "out of device memory";
    case CQG_ERR_CUDA: return "CUDA error";
    case CQG_ERR_TIMEOUT: return "device wait timed out";
    case CQG_ERR_NONFINITE: return "non-finite input";
    case CQG_ERR_STATE: return "invalid call order";
    case CQG_ERR_UNSUPPORTED: return "unsupported input";
  }
  return "unknown status";
}

const char *cqg_class_name(int k) {
  if (!g_names_init) {
    for (int q = 0; q < 55; ++q) {
      int i, j;
      qclass_split(q, i, j);
      snprintf(g_class_names[q], 16, "(%c%c|%c%c)", kLetters[kPairClass[i][0]], kLetters[kPairClass[i][1]],
               kLetters[kPairClass[j][0]], kLetters[kPairClass[j][1]]);
    }
    g_names_init = true;
  }
  if (k < 0 || k >= CQG_NQC) return nullptr;
  return g_class_names[k];
}

cqg_status cqg_create(cqg_ctx **out, int device) {
  if (!out) return CQG_ERR_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return CQG_ERR_CUDA;
  cqg_ctx *ctx = new cqg_ctx();
  ctx->device = device;
  memset(&ctx->stats, 0, sizeof(ctx->stats));
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return CQG_ERR_CUDA;
  }
  // Boys table
  std::vector<double> tab(BOYS_NT * BOYS_NORD);
  for (int i = 0; i < BOYS_NT; ++i) host_boys_row(BOYS_NORD - 1, (long double)i / 10.0L, &tab[i * BOYS_NORD]);
  if (ctx->d_boys.reserve(tab.size()) != cudaSuccess ||
      cudaMemcpy(ctx->d_boys.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete ctx;
    return CQG_ERR_CUDA;
  }
  for (int i = 0; i < 4 + 2 * 55; ++i) cudaEventCreate(&ctx->ev[i]);
  ctx->events = true;
  *out = ctx;
  return CQG_OK;
}

cqg_status cqg_destroy(cqg_ctx *ctx) {
  if (!ctx) return CQG_OK;
  cudaSetDevice(ctx->device);
  ctx->d_center.release(); ctx->d_bf.release(); ctx->d_sz.release();
  ctx->d_pair_sh.release(); ctx->d_pair_Q.release(); ctx->d_pair_poff.release(); ctx->d_pair_np.release();
  ctx->d_prim.release(); ctx->d_boys.release();
  ctx->d_M.release(); ctx->d_Mmax.release(); ctx->d_flags.release();
  ctx->d_cnt.release(); ctx->d_off.release(); ctx->d_range.release(); ctx->d_scan_tmp.release();
  ctx->d_qlist.release(); ctx->d_G.release(); ctx->d_X.release(); ctx->d_AX.release();
  if (ctx->events)
    for (int i = 0; i < 4 + 2 * 55; ++i) cudaEventDestroy(ctx->ev[i]);
  delete ctx;
  return CQG_OK;
}

const char *cqg_last_error(const cqg_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

cqg_status cqg_set_threshold(cqg_ctx *ctx, double thresh) {
  if (!ctx || !(thresh >= 0.0)) return CQG_ERR_BAD_ARG;
  ctx->thresh = thresh;
  return CQG_OK;
}

cqg_status cqg_set_precision(cqg_ctx *ctx, int policy, double cutoff) {
  if (!ctx || (policy != CQG_PREC_FP64 && policy != CQG_PREC_MIXED) || !(cutoff >= 0.0)) return CQG_ERR_BAD_ARG;
  ctx->policy = policy;
  ctx->fp32_cutoff = cutoff;
  return CQG_OK;
}

cqg_status cqg_set_timing(cqg_ctx *ctx, int on) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  ctx->timing = on ? 1 : 0;
  return CQG_OK;
}

cqg_status cqg_get_sizes(cqg_ctx *ctx, int *nshell, int *nbasis, int *maxl) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (nshell) *nshell = ctx->nshell;
  if (nbasis) *nbasis = ctx->nbf;
  if (maxl) *maxl = ctx->maxl;
  return CQG_OK;
}

cqg_status cqg_set_basis(cqg_ctx *ctx, int nshell, const int *L, const int *pure, const int *nprim,
                         const double *alpha, const double *coef, const double *centers) {
  if (!ctx || nshell <= 0 || !L || !pure || !nprim || !alpha || !coef || !centers) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  int tot = 0, maxl = 0;
  for (int s = 0; s < nshell; ++s) {
    if (L[s] < 0 || nprim[s] <= 0) {
      ctx->err = "shell with negative L or no primitives";
      return CQG_ERR_BAD_ARG;
    }
    if (L[s] > CQG_MAXL) {
      ctx->err = "angular momentum above " + std::to_string(CQG_MAXL) + " is not built into this engine";
      return CQG_ERR_UNSUPPORTED;
    }
    if ((pure[s] != 0) != (L[s] > 1)) {
      ctx->err = "engine requires spherical shells exactly for L > 1 (the reference default)";
      return CQG_ERR_UNSUPPORTED;
    }
    tot += nprim[s];
    maxl = std::max(maxl, L[s]);
  }
  ctx->nshell = nshell;
  ctx->maxl = maxl;
  ctx->hL.assign(L, L + nshell);
  ctx->hnprim.assign(nprim, nprim + nshell);
  ctx->halpha.assign(alpha, alpha + tot);
  ctx->hcoef.assign(coef, coef + tot);
  ctx->hcent.assign(centers, centers + 3 * nshell);
  ctx->hbf.resize(nshell);
  ctx->hsz.resize(nshell);
  ctx->hpoff.resize(nshell);
  int f = 0, p = 0;
  for (int s = 0; s < nshell; ++s) {
    ctx->hbf[s] = f;
    ctx->hsz[s] = nfun(L[s]);
    f += ctx->hsz[s];
    ctx->hpoff[s] = p;
    p += nprim[s];
  }
  ctx->nbf = f;
  // shells to device
  std::vector<double3> c3(nshell);
  for (int s = 0; s < nshell; ++s) c3[s] = make_double3(centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]);
  if (ctx->d_center.reserve(nshell) || ctx->d_bf.reserve(nshell) || ctx->d_sz.reserve(nshell)) return CQG_ERR_OOM;
  CUCHK(cudaMemcpy(ctx->d_center.p, c3.data(), nshell * sizeof(double3), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_bf.p, ctx->hbf.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_sz.p, ctx->hsz.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  // pairs by class, internal orientation L_a >= L_b (a >= b when equal L)
  std::vector<std::vector<int2>> bycls(CQG_NPC);
  for (int a = 0; a < nshell; ++a)
    for (int b = 0; b <= a; ++b) {
      int x = a, y = b;
      if (L[y] > L[x]) std::swap(x, y);
      bycls[pair_class_of(L[x], L[y])].push_back(make_int2(x, y));
    }
  ctx->pair_sh.clear();
  for (int c = 0; c < CQG_NPC; ++c) {
    ctx->pc_beg[c] = (int)ctx->pair_sh.size();
    ctx->pair_sh.insert(ctx->pair_sh.end(), bycls[c].begin(), bycls[c].end());
  }
  ctx->pc_beg[CQG_NPC] = (int)ctx->pair_sh.size();
  ctx->pair_Q.assign(ctx->pair_sh.size(), 0.0);
  cqg_status st = upload_pairs(ctx, 0.0);
  if (st != CQG_OK) return st;
  // Schwarz on the device with all primitive pairs (computeSchwartz uses precision 0)
  Pairs P = make_pairs(ctx);
  Shells S = make_shells(ctx);
  double *dQ = ctx->d_pair_Q.p;
  cudaError_t e = cudaSuccess;
  e = e ? e : launch_schwarz<0, 0>(ctx, P, S, ctx->pc_beg[0], ctx->pc_beg[1], dQ);
  e = e ? e : launch_schwarz<1, 0>(ctx, P, S, ctx->pc_beg[1], ctx->pc_beg[2], dQ);
  e = e ? e : launch_schwarz<1, 1>(ctx, P, S, ctx->pc_beg[2], ctx->pc_beg[3], dQ);
  e = e ? e : launch_schwarz<2, 0>(ctx, P, S, ctx->pc_beg[3], ctx->pc_beg[4], dQ);
  e = e ? e : launch_schwarz<2, 1>(ctx, P, S, ctx->pc_beg[4], ctx->pc_beg[5], dQ);
  e = e ? e : launch_schwarz<2, 2>(ctx, P, S, ctx->pc_beg[5], ctx->pc_beg[6], dQ);
  if (e != cudaSuccess) {
    ctx->err = std::string("schwarz kernels: ") + cudaGetErrorString(e);
    return CQG_ERR_CUDA;
  }
  CUCHK(cudaDeviceSynchronize());
  CUCHK(cudaMemcpy(ctx->pair_Q.data(), dQ, ctx->pair_Q.size() * sizeof(double), cudaMemcpyDeviceToHost));
  ctx->Qmat.assign((size_t)nshell * nshell, 0.0);
  for (size_t i = 0; i < ctx->pair_sh.size(); ++i) {
    int a = ctx->pair_sh[i].x, b = ctx->pair_sh[i].y;
    ctx->Qmat[a + (size_t)b * nshell] = ctx->pair_Q[i];
    ctx->Qmat[b + (size_t)a * nshell] = ctx->pair_Q[i];
  }
  // sort each class by Q descending (stable) and rebuild with primitive-pair screening
  for (int c = 0; c < CQG_NPC; ++c) {
    int b0 = ctx->pc_beg[c], b1 = ctx->pc_beg[c + 1];
    std::vector<int> idx(b1 - b0);
    std::iota(idx.begin(), idx.end(), b0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return ctx->pair_Q[x] > ctx->pair_Q[y]; });
    std::vector<int2> sh2;
    std::vector<double> q2;
    for (int i : idx) {
      sh2.push_back(ctx->pair_sh[i]);
      q2.push_back(ctx->pair_Q[i]);
    }
    std::copy(sh2.begin(), sh2.end(), ctx->pair_sh.begin() + b0);
    std::copy(q2.begin(), q2.end(), ctx->pair_Q.begin() + b0);
  }
  st = upload_pairs(ctx, 1e-24);
  if (st != CQG_OK) return st;
  // class-block table
  BlockTable &bt = ctx->bt;
  memset(&bt, 0, sizeof(bt));
  int task = 0;
  for (int k = 0; k < CQG_NQC; ++k) {
    int i, j;
    qclass_split(k, i, j);
    bt.task_beg[k] = task;
    bt.bra_beg[k] = ctx->pc_beg[i];
    bt.ket_beg[k] = ctx->pc_beg[j];
    bt.ket_n[k] = ctx->pc_beg[j + 1] - ctx->pc_beg[j];
    bt.diag[k] = (i == j);
    task += ctx->pc_beg[i + 1] - ctx->pc_beg[i];
  }
  bt.task_beg[CQG_NQC] = task;
  bt.nblk = CQG_NQC;
  ctx->ntask = task;
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (long long *)nullptr, (long long *)nullptr, std::max(task, 1));
  if (ctx->d_cnt.reserve(task + 1) || ctx->d_off.reserve(task + 1) || ctx->d_range.reserve(2 * CQG_NQC) ||
      ctx->d_scan_tmp.reserve(scan_bytes + 16) || ctx->d_M.reserve((size_t)nshell * nshell) ||
      ctx->d_Mmax.reserve(1) || ctx->d_flags.reserve(4))
    return CQG_ERR_OOM;
  return CQG_OK;
}

cqg_status cqg_get_schwarz(cqg_ctx *ctx, double *Q) {
  if (!ctx || !Q) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  memcpy(Q, ctx->Qmat.data(), ctx->Qmat.size() * sizeof(double));
  return CQG_OK;
}

static cqg_status contract_device(cqg_ctx *ctx, int ngroups, const double *const *Xg, double *const *AXg,
                                  const double *sJ, const double *sK, int nx_all, const double *const *Xall,
                                  int ldx, int ldax, cudaStream_t st) {
  const int n = ctx->nbf, nsh = ctx->nshell;
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[0], st));
  // 1. block norms + checks
  XList xl;
  xl.n = nx_all;
  for (int i = 0; i < nx_all; ++i) xl.X[i] = Xall[i];
  CUCHK(cudaMemsetAsync(ctx->d_flags.p, 0, 4 * sizeof(int), st));
  CUCHK(cudaMemsetAsync(ctx->d_Mmax.p, 0, sizeof(double), st));
  {
    dim3 g((nsh + 127) / 128, nsh);
    k_blocknorm<<<g, 128, 0, st>>>(xl, ldx, nsh, ctx->d_bf.p, ctx->d_sz.p, ctx->d_M.p, ctx->d_flags.p, 1e-12);
    CUCHK(cudaGetLastError());
    long long nn = (long long)nsh * nsh;
    int nb = (int)std::min<long long>((nn + 255) / 256, 1184);
    k_maxreduce<<<nb, 256, 0, st>>>(ctx->d_M.p, nn, ctx->d_Mmax.p);
    CUCHK(cudaGetLastError());
  }
  // 2. quartet lists
  Pairs P = make_pairs(ctx);
  {
    int nthr = 256, wpb = nthr / 32;
    int nb = (ctx->ntask + wpb - 1) / wpb;
    k_quartets<false><<<nb, nthr, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, nsh, ctx->d_Mmax.p, ctx->thresh,
                                            ctx->d_cnt.p, nullptr, nullptr);
    CUCHK(cudaGetLastError());
    size_t scan_bytes = ctx->d_scan_tmp.n;
    CUCHK(cub::DeviceScan::ExclusiveSum(ctx->d_scan_tmp.p, scan_bytes, ctx->d_cnt.p, ctx->d_off.p, ctx->ntask, st));
    k_block_ranges<<<1, 64, 0, st>>>(ctx->bt, ctx->d_cnt.p, ctx->d_off.p, ctx->d_range.p);
    CUCHK(cudaGetLastError());
  }
  long long hr[2 * CQG_NQC];
  int hflags[4];
  CUCHK(cudaMemcpyAsync(hr, ctx->d_range.p, sizeof(hr), cudaMemcpyDeviceToHost, st));
  CUCHK(cudaMemcpyAsync(hflags, ctx->d_flags.p, sizeof(hflags), cudaMemcpyDeviceToHost, st));
  CUCHK(cudaStreamSynchronize(st));
  if (hflags[0]) {
    ctx->err = "input density contains NaN or Inf";
    return CQG_ERR_NONFINITE;
  }
  if (hflags[1]) {
    ctx->err = "input matrix is not symmetric; this engine contracts real symmetric X only";
    return CQG_ERR_UNSUPPORTED;
  }
  long long total = hr[2 * CQG_NQC - 1];
  if (ctx->d_qlist.reserve((size_t)std::max<long long>(total, 1)) != cudaSuccess) {
    ctx->err = "quartet list allocation failed";
    return CQG_ERR_OOM;
  }
  {
    int nthr = 256, wpb = nthr / 32;
    int nb = (ctx->ntask + wpb - 1) / wpb;
    k_quartets<true><<<nb, nthr, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, nsh, ctx->d_Mmax.p, ctx->thresh,
                                           nullptr, ctx->d_off.p, ctx->d_qlist.p);
    CUCHK(cudaGetLastError());
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[1], st));
  // 3. ERI + digest per class
  if (ctx->d_G.reserve((size_t)ngroups * n * n) != cudaSuccess) return CQG_ERR_OOM;
  CUCHK(cudaMemsetAsync(ctx->d_G.p, 0, (size_t)ngroups * n * n * sizeof(double), st));
  DigestGroups dg;
  memset(&dg, 0, sizeof(dg));
  dg.ng = ngroups;
  dg.ldx = ldx;
  dg.n = n;
  for (int g = 0; g < ngroups; ++g) {
    dg.X[g] = Xg[g];
    dg.G[g] = ctx->d_G.p + (size_t)g * n * n;
    dg.sJ[g] = sJ[g];
    dg.sK[g] = sK[g];
  }
  memset(ctx->stats.class_quartets, 0, sizeof(ctx->stats.class_quartets));
  memset(ctx->stats.class_ms, 0, sizeof(ctx->stats.class_ms));
  double mflops = 0;
  long long nprimq = 0;
  for (int k = 0; k < CQG_NQC; ++k) {
    long long nq = hr[2 * k + 1] - hr[2 * k];
    ctx->stats.class_quartets[k] = nq;
    int i, j;
    qclass_split(k, i, j);
    (void)i;
    (void)j;
    if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[4 + 2 * k], st));
    cudaError_t e = kEriLaunch[k](ctx, k, nq, st, dg);
    if (e != cudaSuccess) {
      ctx->err = std::string("eri kernel ") + cqg_class_name(k) + ": " + cudaGetErrorString(e);
      return CQG_ERR_CUDA;
    }
    if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[5 + 2 * k], st));
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[2], st));
  // 4. AX += 0.5 (Gh + Gh^T)
  for (int g = 0; g < ngroups; ++g) {
    dim3 grid((n + 31) / 32, (n + 31) / 32), blk(32, 8);
    k_finalize<<<grid, blk, 0, st>>>(dg.G[g], n, AXg[g], ldax);
    CUCHK(cudaGetLastError());
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[3], st));
  ctx->stats.quartets = total;
  ctx->stats.quartets_fp32 = 0;
  (void)mflops;
  (void)nprimq;
  return CQG_OK;
}

// group (X, AX) pairs and fold scales: COULOMB -> sJ, EXCHANGE -> sK
static cqg_status plan_groups(cqg_ctx *ctx, int nmat, const double *const *X, double *const *AX, const int *types,
                              const double *scale, int &ng, const double **Xg, double **AXg, double *sJ, double *sK,
                              int &nxu, const double **Xu) {
  ng = 0;
  nxu = 0;
  for (int i = 0; i < nmat; ++i) {
    if (!X[i] || !AX[i] || (types[i] != CQG_COULOMB && types[i] != CQG_EXCHANGE)) {
      ctx->err = "null matrix or unknown contraction type";
      return CQG_ERR_BAD_ARG;
    }
    bool seen = false;
    for (int u = 0; u < nxu; ++u)
      if (Xu[u] == X[i]) seen = true;
    if (!seen) {
      if (nxu >= 8) return CQG_ERR_BAD_ARG;
      Xu[nxu++] = X[i];
    }
    int g = -1;
    for (int k = 0; k < ng; ++k)
      if (Xg[k] == X[i] && AXg[k] == AX[i]) g = k;
    if (g < 0) {
      if (ng >= CQG_MAXG) {
        ctx->err = "too many distinct (X, AX) pairs in one call";
        return CQG_ERR_UNSUPPORTED;
      }
      g = ng++;
      Xg[g] = X[i];
      AXg[g] = AX[i];
      sJ[g] = sK[g] = 0.0;
    }
    if (types[i] == CQG_COULOMB) sJ[g] += scale[i];
    else sK[g] += scale[i];
  }
  return CQG_OK;
}

cqg_status cqg_twoe_contract_direct(cqg_ctx *ctx, int nmat, const double *const *X, double *const *AX,
                                    const int *types, const double *scale, int ld, int on_device, void *stream) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  if (nmat <= 0 || nmat > 8 || !X || !AX || !types || !scale || ld < ctx->nbf) {
    ctx->err = "bad list sizes or leading dimension";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const double *Xg[CQG_MAXG];
  double *AXg[CQG_MAXG];
  double sJ[CQG_MAXG], sK[CQG_MAXG];
  const double *Xu[8];
  int ng, nxu;
  cqg_status s = plan_groups(ctx, nmat, X, AX, types, scale, ng, Xg, AXg, sJ, sK, nxu, Xu);
  if (s != CQG_OK) return s;
  const int n = ctx->nbf;
  if (on_device) return contract_device(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ld, ld, st);
  // host pointers: stage distinct X and each group's AX on the device
  size_t nn = (size_t)n * n;
  if (ctx->d_X.reserve(nn * nxu) || ctx->d_AX.reserve(nn * ng)) return CQG_ERR_OOM;
  const double *dXu[8];
  for (int u = 0; u < nxu; ++u) {
    dXu[u] = ctx->d_X.p + nn * u;
    CUCHK(cudaMemcpy2DAsync((void *)dXu[u], n * sizeof(double), Xu[u], ld * sizeof(double), n * sizeof(double), n,
                            cudaMemcpyHostToDevice, st));
  }
  const double *dXg[CQG_MAXG];
  double *dAXg[CQG_MAXG];
  for (int g = 0; g < ng; ++g) {
    for (int u = 0; u < nxu; ++u)
      if (Xu[u] == Xg[g]) dXg[g] = dXu[u];
    dAXg[g] = ctx->d_AX.p + nn * g;
    CUCHK(cudaMemcpy2DAsync(dAXg[g], n * sizeof(double), AXg[g], ld * sizeof(double), n * sizeof(double), n,
                            cudaMemcpyHostToDevice, st));
  }
  s = contract_device(ctx, ng, dXg, dAXg, sJ, sK, nxu, dXu, n, n, st);
  if (s != CQG_OK) return s;
  for (int g = 0; g < ng; ++g)
    CUCHK(cudaMemcpy2DAsync(AXg[g], ld * sizeof(double), dAXg[g], n * sizeof(double), n * sizeof(double), n,
                            cudaMemcpyDeviceToHost, st));
  CUCHK(cudaStreamSynchronize(st));
  return CQG_OK;
}

cqg_status cqg_form_pt(cqg_ctx *ctx, int is_rhf, double xHF, const double *Ps, const double *Pz, double *PTs,
                       double *PTz, int ld, int on_device, void *stream) {
  if (!ctx || !Ps || !PTs || (!is_rhf && (!Pz || !PTz))) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int n = ctx->nbf;
  // PT zeroed first (singleslater_fock.h:47,54)
  if (on_device) {
    CUCHK(cudaMemset2DAsync(PTs, ld * sizeof(double), 0, n * sizeof(double), n, st));
    if (!is_rhf) CUCHK(cudaMemset2DAsync(PTz, ld * sizeof(double), 0, n * sizeof(double), n, st));
  } else {
    for (int c = 0; c < n; ++c) memset(PTs + (size_t)c * ld, 0, n * sizeof(double));
    if (!is_rhf)
      for (int c = 0; c < n; ++c) memset(PTz + (size_t)c * ld, 0, n * sizeof(double));
  }
  if (is_rhf) {
    const double *X[2] = {Ps, Ps};
    double *AX[2] = {PTs, PTs};
    int types[2] = {CQG_COULOMB, CQG_EXCHANGE};
    double scale[2] = {1.0, xHF};
    return cqg_twoe_contract_direct(ctx, 2, X, AX, types, scale, ld, on_device, stream);
  }
  const double *X[3] = {Ps, Ps, Pz};
  double *AX[3] = {PTs, PTs, PTz};
  int types[3] = {CQG_COULOMB, CQG_EXCHANGE, CQG_EXCHANGE};
  double scale[3] = {1.0, xHF, xHF};
  return cqg_twoe_contract_direct(ctx, 3, X, AX, types, scale, ld, on_device, stream);
}

cqg_status cqg_get_stats(cqg_ctx *ctx, cqg_stats *out) {
  if (!ctx || !out) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  CUCHK(cudaDeviceSynchronize());
  cqg_stats &s = ctx->stats;
  double mf = 0;
  for (int k = 0; k < CQG_NQC; ++k) {
    int i, j;
    qclass_split(k, i, j);
    int la = kPairClass[i][0], lb = kPairClass[i][1], lc = kPairClass[j][0], ld = kPairClass[j][1];
    (void)la;
    mf += (double)s.class_quartets[k] * md_v1_digest_flops(la, lb, lc, ld);
  }
  (void)mf;
  if (ctx->timing) {
    float ms;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    s.ms_screen = ms;
    cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
    s.ms_eri = ms;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[3]);
    s.ms_total = ms;
    for (int k = 0; k < CQG_NQC; ++k) {
      if (s.class_quartets[k] > 0) {
        cudaEventElapsedTime(&ms, ctx->ev[4 + 2 * k], ctx->ev[5 + 2 * k]);
        s.class_ms[k] = ms;
      }
    }
  }
  *out = s;
  return CQG_OK;
}

cqg_status cqg_probe_fma_peak(int device, int fp64, double ms_target, double *tflops) {
  if (!tflops) return CQG_ERR_BAD_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return CQG_ERR_CUDA;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  void *buf = nullptr;
  if (cudaMalloc(&buf, 64) != cudaSuccess) return CQG_ERR_OOM;
  int blocks = nsm * 8, threads = 256, iters = 256;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float ms = 0;
  for (int rep = 0; rep < 8; ++rep) {
    cudaEventRecord(a);
    if (fp64) k_fma_probe<double><<<blocks, threads>>>((double *)buf, iters, 1.0);
    else k_fma_probe<float><<<blocks, threads>>>((float *)buf, iters, 1.0f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    if (ms < ms_target && rep < 7) iters = (int)std::min(1 << 24, (int)(iters * std::max(1.5, ms_target / std::max(ms, 0.01f))));
    else break;
  }
  double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(buf);
  return cudaGetLastError() == cudaSuccess ? CQG_OK : CQG_ERR_CUDA;
}

}  // extern "C"
