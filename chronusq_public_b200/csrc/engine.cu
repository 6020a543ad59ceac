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
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/cqgpu.h"
#include "eri_common.cuh"
#include "_gen/eri_classes.cuh"
#include "eri_warp.cuh"
#include "one_e.cuh"

#define CQG_MAXL 3
#define CQG_NPC ((CQG_MAXL + 1) * (CQG_MAXL + 2) / 2)       // pair classes
#define CQG_NQC (CQG_NPC * (CQG_NPC + 1) / 2)                // quartet classes
#define CQG_MAXG 4
#define CQG_NBUCKET 16

static_assert(CQG_NQC <= 55, "class table");

// ------------------------------------------------------------------ class tables ---
static_assert(CQG_GEN_MAXL == CQG_MAXL, "generated ERI code must match CQG_MAXL");
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
  const int *bf;     // first basis function of the shell within its molecule
  const int *mol;    // molecule of the shell
};

// Per-molecule layout: a context holds nmol >= 1 molecules (a batch).  Matrices of
// molecule m are packed at offset xoff[m] with leading dimension nbf[m]; with a single
// molecule the caller's matrices are used in place (xoff[0] = 0, leading dimension ldx).
struct Mols {
  int nmol;
  const int *shoff;              // first (global) shell of molecule m
  const int *nsh;                // shells of molecule m
  const long long *Moff;         // offset of molecule m's nsh_m x nsh_m block-norm matrix
  const long long *xoff;         // offset of molecule m's matrices in packed storage
  const int *nbf;                // basis functions of molecule m
  const unsigned char *active;   // molecule m takes part in the call
  const int *molbk;              // [m][ket pair class][bucket + 1]: first pair of each bucket
};
struct Pairs {
  const int2 *sh;       // (shell a, shell b), internal orientation L_a >= L_b
  const double *Q;      // Schwarz bound
  const int *poff;      // first primitive pair
  const int *np;        // number of primitive pairs (after primitive screening)
  const int *kk;        // nprim(a) * nprim(b) of the contracted shells (model count)
  const PrimPair *prim;
};
struct DigestGroups {
  const double *X[CQG_MAXG];
  double *G[CQG_MAXG];
  double sJ[CQG_MAXG];
  double sK[CQG_MAXG];
  int ng;
  int ldx;                        // leading dimension of X when nmol == 1
  int batch;                      // matrices are packed per molecule (Mols.xoff / nbf)
  const long long *xoff;
  const int *nbf;
};

// base pointers and leading dimensions of molecule m's X and Gh
__device__ __forceinline__ void mol_view(const DigestGroups &dg, int g, int m, const double *&X, double *&G,
                                         size_t &ldx, size_t &ldg) {
  if (dg.batch) {
    const long long o = dg.xoff[m];
    X = dg.X[g] + o;
    G = dg.G[g] + o;
    ldx = ldg = (size_t)dg.nbf[m];
  } else {
    X = dg.X[g];
    G = dg.G[g];
    ldx = dg.ldx;
    ldg = (size_t)dg.nbf[0];
  }
}

// ------------------------------------------------------------------ kernels ---
// Schwarz: Q(ab) = sqrt(max_ij |(ij|ij)|) for pairs [beg, end) of one class.
template <int LA, int LB>
__global__ void __launch_bounds__(128) k_schwarz(Pairs P, Shells S, const double *__restrict__ boys_g,
                                                 int beg, int end, double *__restrict__ Qout) {
  __shared__ __align__(16) double boys[BOYS_NT * BOYS_SROW];
  stage_boys<2 * (LA + LB)>(boys_g, boys);
  __syncthreads();
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
__global__ void k_blocknorm(XList xl, int ldx, Mols mols, const int *__restrict__ bf,
                            const int *__restrict__ sz, double *__restrict__ M, double *__restrict__ MT,
                            int *__restrict__ flags, double sym_tol) {
  const int mol = blockIdx.z;
  const int nsh = mols.nsh[mol];
  int s1 = blockIdx.x * blockDim.x + threadIdx.x;
  int s2 = blockIdx.y;
  if (s1 >= nsh || s2 >= nsh) return;
  double *Mm = M + mols.Moff[mol];
  double *MTm = MT + mols.Moff[mol];
  if (!mols.active[mol]) {
    Mm[(size_t)s1 + (size_t)s2 * nsh] = 0.0;
    MTm[(size_t)s2 + (size_t)s1 * nsh] = 0.0;
    return;
  }
  const int g1 = mols.shoff[mol] + s1, g2 = mols.shoff[mol] + s2;
  int r0 = bf[g1], c0 = bf[g2], nr = sz[g1], nc = sz[g2];
  if (mols.nmol > 1) ldx = mols.nbf[mol];
  const long long xo = mols.nmol > 1 ? mols.xoff[mol] : 0;
  double mx = 0.0;
  int bad = 0, asym = 0;
  for (int m = 0; m < xl.n; ++m) {
    const double *X = xl.X[m] + xo;
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
  Mm[(size_t)s1 + (size_t)s2 * nsh] = mx;
  MTm[(size_t)s2 + (size_t)s1 * nsh] = mx;   // transposed copy: M(s1, .) as a contiguous column
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
  int ket_class[CQG_NQC];      // pair class of the ket
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

// Density-weighted Schwarz bound of a quartet: max of the six shell-block norms of the
// density times Q_ab Q_cd (contract.h:112-131).  The four norms that pair a bra shell with
// a ket shell are read from the transposed copy MT, where M(s1, .) and M(s2, .) are the
// contiguous columns s1 and s2 (one pair of columns per bra pair, so they stay in L1);
// m12 = M(s1, s2) is the bra's own, the same for every ket.
__device__ __forceinline__ double quartet_bound(const double *__restrict__ M, const double *__restrict__ col1,
                                                const double *__restrict__ col2, double m12, int nsh, int shoff,
                                                int2 cd, double qab, double qcd) {
  const int s3 = cd.x - shoff, s4 = cd.y - shoff;
  double m = fmax(m12, col1[s4]);
  m = fmax(m, col2[s4]);
  m = fmax(m, M[s3 + (size_t)s4 * nsh]);
  m = fmax(m, col1[s3]);
  m = fmax(m, col2[s3]);
  return m * qab * qcd;
}

// Count (FILL=false) or write (FILL=true) the passing quartets of each task.  One warp
// per task; ket pairs scanned in ascending order, survivors compacted with a ballot so
// the list is deterministic.  Quartets whose bound is below `cut32` go to the FP32 list
// (counts cnt[ntask + task], offsets off[ntask + task]); the rest to the FP64 list.
template <bool FILL>
__global__ void __launch_bounds__(256) k_quartets(BlockTable bt, int ntask, Pairs P, const double *__restrict__ M,
                                                  const double *__restrict__ MT, Mols mols, const int *__restrict__ shmol,
                                                  const double *__restrict__ Mmax, double thresh,
                                                  double cut32, long long *__restrict__ cnt,
                                                  const long long *__restrict__ off, uint2 *__restrict__ qlist,
                                                  unsigned long long *__restrict__ blkacc, long long vt0,
                                                  long long vt1, long long obase, long long cap) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ntask) return;
  // fill pass: only the FP64 (virtual task warp) and FP32 (ntask + warp) parts inside the chunk
  const bool do64 = !FILL || (warp >= vt0 && warp < vt1);
  const bool do32 = !FILL || (ntask + warp >= vt0 && ntask + warp < vt1);
  if (FILL && !do64 && !do32) return;
  int blk = find_block(bt, warp);
  int bra = bt.bra_beg[blk] + (warp - bt.task_beg[blk]);
  double qb = P.Q[bra];
  double mm = *Mmax;
  double cut = (qb * mm > 0.0) ? thresh / (qb * mm) * (1.0 - 1e-12) : 0.0;
  int2 ab = P.sh[bra];
  const int mol = shmol[ab.x];
  const int nsh = mols.nsh[mol], shoff = mols.shoff[mol];
  const double *Mm = M + mols.Moff[mol];
  const double *col1 = MT + mols.Moff[mol] + (size_t)(ab.x - shoff) * nsh;
  const double *col2 = MT + mols.Moff[mol] + (size_t)(ab.y - shoff) * nsh;
  const double m12 = Mm[(ab.x - shoff) + (size_t)(ab.y - shoff) * nsh];
  const int *bkt = mols.molbk + ((size_t)mol * CQG_NPC + bt.ket_class[blk]) * (CQG_NBUCKET + 1);
  const long long base64 = FILL ? off[warp] - obase : 0, base32 = FILL ? off[ntask + warp] - obase : 0;
  long long c64 = 0, c32 = 0;
  unsigned long long km64 = 0, ke64 = 0, km32 = 0, ke32 = 0;
  if (qb * mm > 0.0 && mols.active[mol]) {
    for (int bk = 0; bk < CQG_NBUCKET; ++bk) {
      const int kb = bkt[bk], ke = bkt[bk + 1];
      if (ke <= kb) continue;
      int kend = kb + coarse_range(P.Q, kb, ke - kb, cut);
      if (bt.diag[blk]) kend = min(kend, bra + 1);   // unique pairs of pairs: ket <= bra
      for (int k0 = kb; k0 < kend; k0 += 32) {
        int ket = k0 + lane;
        bool pass = false, lo = false;
        if (ket < kend) {
          const double bnd = quartet_bound(Mm, col1, col2, m12, nsh, shoff, P.sh[ket], qb, P.Q[ket]);
          pass = bnd >= thresh;
          lo = pass && bnd < cut32;
        }
        const bool hi = pass && !lo;
        unsigned b64 = __ballot_sync(0xffffffffu, hi), b32 = __ballot_sync(0xffffffffu, lo);
        const unsigned below = (1u << lane) - 1u;
        if (FILL && hi && do64) {
          const long long pos = base64 + c64 + __popc(b64 & below);
          if (pos < cap) qlist[pos] = make_uint2((unsigned)bra, (unsigned)ket);
        }
        if (FILL && lo && do32) {
          const long long pos = base32 + c32 + __popc(b32 & below);
          if (pos < cap) qlist[pos] = make_uint2((unsigned)bra, (unsigned)ket);
        }
        if (!FILL && hi) {
          km64 += (unsigned long long)P.kk[ket];
          ke64 += (unsigned long long)P.np[ket];
        }
        if (!FILL && lo) {
          km32 += (unsigned long long)P.kk[ket];
          ke32 += (unsigned long long)P.np[ket];
        }
        c64 += __popc(b64);
        c32 += __popc(b32);
      }
    }
  }
  if (!FILL) {
    for (int o = 16; o > 0; o >>= 1) {
      km64 += __shfl_xor_sync(0xffffffffu, km64, o);
      ke64 += __shfl_xor_sync(0xffffffffu, ke64, o);
      km32 += __shfl_xor_sync(0xffffffffu, km32, o);
      ke32 += __shfl_xor_sync(0xffffffffu, ke32, o);
    }
    if (lane == 0) {
      cnt[warp] = c64;
      cnt[ntask + warp] = c32;
      if (c64) {
        atomicAdd(blkacc + 4 * blk + 0, km64 * (unsigned long long)P.kk[bra]);
        atomicAdd(blkacc + 4 * blk + 1, ke64 * (unsigned long long)P.np[bra]);
      }
      if (c32) {
        atomicAdd(blkacc + 4 * blk + 2, km32 * (unsigned long long)P.kk[bra]);
        atomicAdd(blkacc + 4 * blk + 3, ke32 * (unsigned long long)P.np[bra]);
      }
    }
  }
}

// Ranges [beg, end) of the quartet list per (precision, class block) from the per-task
// counts and offsets; virtual block b = prec * nblk + block, prec 0 = FP64, 1 = FP32.
__global__ void k_block_ranges(BlockTable bt, int ntask, const long long *__restrict__ cnt,
                               const long long *__restrict__ off, long long *__restrict__ range, long long cap,
                               int *__restrict__ flags) {
  int vb = threadIdx.x;
  if (vb == 0 && ntask > 0 && off[2 * ntask - 1] + cnt[2 * ntask - 1] > cap) flags[2] = 1;   // list overflow
  if (vb >= 2 * bt.nblk) return;
  const int prec = vb / bt.nblk, b = vb % bt.nblk;
  const int t0 = prec * ntask + bt.task_beg[b], t1 = prec * ntask + bt.task_beg[b + 1];
  long long beg = 0, end = 0;
  if (t1 > t0) {
    beg = off[t0];
    end = off[t1 - 1] + cnt[t1 - 1];
  } else if (t0 > 0) {
    beg = end = off[t0 - 1] + cnt[t0 - 1];
  }
  range[2 * vb] = min(beg, cap);
  range[2 * vb + 1] = min(end, cap);
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// J/K digest of one quartet (contract.h:145-171), half of the updates:
//   COULOMB : Gh(a,b) += sJ sum_cd X(d,c) v ;  Gh(c,d) += sJ sum_ab X(b,a) v
//   EXCHANGE: Gh(a,c) += sK X(b,d) v ; Gh(b,d) += sK X(a,c) v ; Gh(a,d) += sK X(b,c) v ;
//             Gh(b,c) += sK X(a,d) v
// with v = (ab|cd) * degeneracy, sK = 0.5 * scale_K; the other half is Gh^T (added in
// k_finalize).  All lanes of the warp call this; `valid` lanes hold a quartet, and when
// every lane shares the bra pair (`bra_uniform`) the Gh(a,b) sums are reduced across the
// warp before one atomic per element.
template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void digest(const double *v, double deg, int a0, int b0, int c0, int d0,
                                       const DigestGroups &dg, bool valid, bool bra_uniform, int mol) {
  const int lane = threadIdx.x & 31;
  for (int g = 0; g < dg.ng; ++g) {
    const double *Xv;
    double *G;
    size_t ld, n;
    mol_view(dg, g, mol, Xv, G, ld, n);
    const double *__restrict__ X = Xv;
    const double sJ = dg.sJ[g] * deg;
    const double sK = 0.5 * dg.sK[g] * deg;
    if (dg.sJ[g] != 0.0) {
      double xdc[NC * ND], xba[NA * NB];
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) xdc[c * ND + d] = valid ? __ldg(X + (d0 + d) + (c0 + c) * ld) : 0.0;
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) xba[a * NB + b] = valid ? __ldg(X + (b0 + b) + (a0 + a) * ld) : 0.0;
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          double s = 0.0;
#pragma unroll
          for (int cd = 0; cd < NC * ND; ++cd) s += xdc[cd] * v[(a * NB + b) * NC * ND + cd];
          s *= sJ;
          if (bra_uniform) {
            s = warp_sum(s);
            if (lane == 0) atomicAdd(G + (a0 + a) + (b0 + b) * n, s);
          } else if (valid) {
            atomicAdd(G + (a0 + a) + (b0 + b) * n, s);
          }
        }
      if (valid) {
#pragma unroll
        for (int cd = 0; cd < NC * ND; ++cd) {
          double s = 0.0;
#pragma unroll
          for (int ab = 0; ab < NA * NB; ++ab) s += xba[ab] * v[ab * NC * ND + cd];
          atomicAdd(G + (c0 + cd / ND) + (d0 + cd % ND) * n, sJ * s);
        }
      }
    }
    // Exchange updates go to Gh(c, a), Gh(d, b), Gh(d, a), Gh(c, b): k_finalize adds
    // (Gh + Gh^T) / 2, so either orientation gives the same result, and with the bra
    // index (the same across a bra-uniform warp) as the column the lanes' atomics land in
    // one column of Gh.
    if (dg.sK[g] != 0.0 && valid) {
      // X is symmetric (checked on entry): its exchange blocks are read as X(d, b), X(c, a),
      // X(c, b), X(d, a), with the bra index (the same across a bra-uniform warp) as the column
      double xbd[NB * ND], xac[NA * NC], xbc[NB * NC], xad[NA * ND];
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int d = 0; d < ND; ++d) xbd[b * ND + d] = __ldg(X + (d0 + d) + (b0 + b) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) xac[a * NC + c] = __ldg(X + (c0 + c) + (a0 + a) * ld);
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) xbc[b * NC + c] = __ldg(X + (c0 + c) + (b0 + b) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int d = 0; d < ND; ++d) xad[a * ND + d] = __ldg(X + (d0 + d) + (a0 + a) * ld);
#pragma unroll
      for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int d = 0; d < ND; ++d) s += xbd[b * ND + d] * v[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (c0 + c) + (a0 + a) * n, sK * s);
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
          atomicAdd(G + (d0 + d) + (b0 + b) * n, sK * s);
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
          atomicAdd(G + (d0 + d) + (a0 + a) * n, sK * s);
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
          atomicAdd(G + (c0 + c) + (b0 + b) * n, sK * s);
        }
    }
  }
}

template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_jk_one(const uint2 *__restrict__ ql, long long i, long long wfirst, long long end,
                                           const Pairs &P, const Shells &S, const double *boys,
                                           const DigestGroups &dg);

// Per-thread class kernel: persistent grid over the class's quartet range; the Boys rows
// of this class are staged in shared memory once per block.  T is the arithmetic type of
// everything after the (FP64) Boys values; the digest accumulates in FP64.
// Threads per block of the per-thread class kernels (each block stages its own copy of the
// Boys rows in shared memory).  128 and 256 measure within 2 % of each other on (H2O)_32
// cc-pVDZ; 512 caps registers at 128 and spills in the p/d classes.
#ifndef CQG_ERI_THREADS
#define CQG_ERI_THREADS 128
#endif
constexpr int kEriThreads = CQG_ERI_THREADS;

template <int LA, int LB, int LC, int LD, typename T>
__global__ void __launch_bounds__(kEriThreads) k_eri_jk(const uint2 *__restrict__ ql, const long long *__restrict__ range,
                                                int blk, Pairs P, Shells S, const double *__restrict__ boys_g,
                                                DigestGroups dg) {
  __shared__ __align__(16) double boys[BOYS_NT * BOYS_SROW];
  stage_boys<LA + LB + LC + LD>(boys_g, boys);
  __syncthreads();
  const long long beg = range[2 * blk], end = range[2 * blk + 1];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = beg + blockIdx.x * (long long)blockDim.x + threadIdx.x;; i += stride) {
    const long long wfirst = i - (threadIdx.x & 31);
    if (wfirst >= end) return;   // the whole warp is past the end of the class
    eri_jk_one<LA, LB, LC, LD, T>(ql, i, wfirst, end, P, S, boys, dg);
  }
}

template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_jk_one(const uint2 *__restrict__ ql, long long i, long long wfirst, long long end,
                                           const Pairs &P, const Shells &S, const double *boys,
                                           const DigestGroups &dg) {
  const bool valid = i < end;
  constexpr int NA = nfun_c(LA), NB = nfun_c(LB), NC = nfun_c(LC), ND = nfun_c(LD);
  const uint2 e = ql[valid ? i : wfirst];
  const int2 ab = P.sh[e.x], cd = P.sh[e.y];
  double v[NA * NB * NC * ND];
  if (valid) {
    const double3 A = S.center[ab.x], B = S.center[ab.y], C = S.center[cd.x], D = S.center[cd.y];
    if constexpr (sizeof(T) == sizeof(double)) {
      EriClass<LA, LB, LC, LD>::template run<double>(P.prim + P.poff[e.x], P.np[e.x], P.prim + P.poff[e.y],
                                                     P.np[e.y], A, B, C, D, boys, v);
    } else {
      T vt[NA * NB * NC * ND];
      EriClass<LA, LB, LC, LD>::template run<T>(P.prim + P.poff[e.x], P.np[e.x], P.prim + P.poff[e.y], P.np[e.y],
                                                A, B, C, D, boys, vt);
#pragma unroll
      for (int k = 0; k < NA * NB * NC * ND; ++k) v[k] = (double)vt[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < NA * NB * NC * ND; ++k) v[k] = 0.0;
  }
  const unsigned bra0 = __shfl_sync(0xffffffffu, e.x, 0);
  const bool uniform = __all_sync(0xffffffffu, e.x == bra0);
  const double deg = (ab.x == ab.y ? 1.0 : 2.0) * (cd.x == cd.y ? 1.0 : 2.0) * (e.x == e.y ? 1.0 : 2.0);
  digest<NA, NB, NC, ND>(v, deg, S.bf[ab.x], S.bf[ab.y], S.bf[cd.x], S.bf[cd.y], dg, valid, uniform, S.mol[ab.x]);
}

// ------------------------------------------------------------- warp-mode classes ---
// SCHWARZ = false: quartets from the list, J/K digest.  SCHWARZ = true: "quartet" i is
// pair i with itself, and the kernel writes Q(i) = sqrt(max |(ab|ab)| diagonal).
// One FP64 tensor-core step D += A B on an 8x8x4 tile (mma.sync m8n8k4 .f64).  Fragments:
// a = A[g][t], b = B[t][g], d[i] = D[g][2t+i] with g = lane / 4, t = lane % 4.
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Whether a warp class runs its two Hermite contractions on the FP64 tensor cores:
//   W[h][cd] += sum_k R[h + k] KC[k][cd]     (per primitive quartet; KC = signed ket E products)
//   C[ab][cd] += sum_h EB[ab][h] W[h][cd]    (per bra primitive pair)
// W's 8x8 tiles are held in registers across the ket loop, so classes with more than 25
// tiles keep the shared-memory loops.  FP32 lists use the same FP64 tiles: their R and E
// values are FP32 and the products are accumulated in FP64.
template <int LA, int LB, int LC, int LD, bool SCHWARZ, typename T>
struct WarpMma {
  static constexpr int HP = warpmd::nherm(LA + LB), HQ = warpmd::nherm(LC + LD);
  static constexpr int NCCD = warpmd::ncart(LC) * warpmd::ncart(LD), NCAB = warpmd::ncart(LA) * warpmd::ncart(LB);
  static constexpr int MT = (HP + 7) / 8, NT = (NCCD + 7) / 8, KT = (HQ + 3) / 4;
  static constexpr int MTC = (NCAB + 7) / 8, KTH = (HP + 3) / 4;
  static constexpr bool on = !SCHWARZ && MT * NT <= 25;
  // larger classes accumulate W in shared memory, NTB column tiles at a time
  static constexpr bool onS = !SCHWARZ && !on;
  static constexpr int NTB = MT >= 25 ? 1 : 25 / MT;
  static constexpr bool any = on || onS;
};

template <int LA, int LB, int LC, int LD, bool SCHWARZ, typename T>
__global__ void __launch_bounds__(128) k_eri_jk_warp(const uint2 *__restrict__ ql, const long long *__restrict__ range,
                                                     int blk, long long sbeg, long long send, Pairs P, Shells S,
                                                     const double *__restrict__ boys, DigestGroups dg,
                                                     double *__restrict__ Qout) {
  using WD = warpmd::WarpDims<LA, LB, LC, LD>;
  constexpr int L = WD::L, NCCD = WD::NCCD;
  constexpr int NBUF = (WD::NW > WD::NC) ? WD::NW : WD::NC;
  extern __shared__ double smem[];
  // decode tables: Hermite (t,u,v) of index h, and Cartesian exponents of bra / ket pairs,
  // packed 4 bits per exponent
  __shared__ int s_h[WD::HL];
  __shared__ int s_cab[WD::NCAB];
  __shared__ int s_ccd[NCCD];
  using MM = WarpMma<LA, LB, LC, LD, SCHWARZ, T>;
  // s_sum[h * HQ + k]: index of the Hermite triple h + k (bra h, ket k) in R
  __shared__ short s_sum[MM::any ? MM::HP * MM::HQ : 1];
  if constexpr (MM::any) {
    for (int k = threadIdx.x; k < MM::HP * MM::HQ; k += blockDim.x) {
      int t1, u1, v1, t2, u2, v2;
      warpmd::herm_of(k / MM::HQ, t1, u1, v1);
      warpmd::herm_of(k % MM::HQ, t2, u2, v2);
      s_sum[k] = (short)warpmd::hidx(t1 + t2, u1 + u2, v1 + v2);
    }
  }
  // s_rec[h], h >= 1: the downward recursion R^n_h = P_d R^{n+1}_a + m R^{n+1}_b of Hermite
  // triple h, packed as a | b << 10 | d << 20 | m << 22 (d = 0, 1, 2 for x, y, z)
  __shared__ int s_rec[WD::HL];
  for (int k = threadIdx.x; k < WD::HL; k += blockDim.x) {
    int t, u, v;
    warpmd::herm_of(k, t, u, v);
    s_h[k] = t | (u << 4) | (v << 8);
    int a = 0, b = 0, d = 0, m = 0;
    if (t > 0) {
      a = warpmd::hidx(t - 1, u, v);
      if (t > 1) b = warpmd::hidx(t - 2, u, v), m = t - 1;
    } else if (u > 0) {
      d = 1;
      a = warpmd::hidx(t, u - 1, v);
      if (u > 1) b = warpmd::hidx(t, u - 2, v), m = u - 1;
    } else if (v > 0) {
      d = 2;
      a = warpmd::hidx(t, u, v - 1);
      if (v > 1) b = warpmd::hidx(t, u, v - 2), m = v - 1;
    }
    s_rec[k] = a | (b << 10) | (d << 20) | (m << 22);
  }
  for (int k = threadIdx.x; k < WD::NCAB; k += blockDim.x) {
    int x0, y0, z0, x1, y1, z1;
    warpmd::cart_of(LA, k / warpmd::ncart(LB), x0, y0, z0);
    warpmd::cart_of(LB, k % warpmd::ncart(LB), x1, y1, z1);
    s_cab[k] = x0 | (y0 << 4) | (z0 << 8) | (x1 << 12) | (y1 << 16) | (z1 << 20);
  }
  for (int k = threadIdx.x; k < NCCD; k += blockDim.x) {
    int x0, y0, z0, x1, y1, z1;
    warpmd::cart_of(LC, k / warpmd::ncart(LD), x0, y0, z0);
    warpmd::cart_of(LD, k % warpmd::ncart(LD), x1, y1, z1);
    s_ccd[k] = x0 | (y0 << 4) | (z0 << 8) | (x1 << 12) | (y1 << 16) | (z1 << 20);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // per warp: staged density blocks (double) then the T work arrays
  constexpr size_t WARP_BYTES = sizeof(double) * WD::NXS + sizeof(T) * (3 * WD::NEB + 3 * WD::NEK + 2 * WD::HL + 2 * NBUF);
  constexpr size_t WARP_STRIDE = (WARP_BYTES + 15) / 16 * 16;
  double *Xs = reinterpret_cast<double *>(reinterpret_cast<char *>(smem) + wid * WARP_STRIDE);
  T *Eb = reinterpret_cast<T *>(Xs + WD::NXS);
  T *Ek = Eb + 3 * WD::NEB;
  T *Ra = Ek + 3 * WD::NEK;
  T *Rb = Ra + WD::HL;
  T *W = Rb + WD::HL;
  T *Cc = W + NBUF;
  long long beg, end;
  if (SCHWARZ) {
    beg = sbeg;
    end = send;
  } else {
    beg = range[2 * blk];
    end = range[2 * blk + 1];
  }
  const long long stride = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long q = beg + (long long)blockIdx.x * (blockDim.x >> 5) + wid; q < end; q += stride) {
    uint2 e;
    if (SCHWARZ) e = make_uint2((unsigned)q, (unsigned)q);
    else e = ql[q];
    const int2 ab = P.sh[e.x], cdp = P.sh[e.y];
    const double3 A = S.center[ab.x], B = S.center[ab.y], C = S.center[cdp.x], D = S.center[cdp.y];
    const PrimPair *pbp = P.prim + P.poff[e.x];
    const PrimPair *pkp = P.prim + P.poff[e.y];
    const int nb = P.np[e.x], nk = P.np[e.y];
    __syncwarp();
    for (int k = lane; k < WD::NC; k += 32) Cc[k] = T(0);
    for (int ib = 0; ib < nb; ++ib) {
      const PrimPair bp = pbp[ib];
      __syncwarp();
      if (lane < 3) {
        const double Pc = lane == 0 ? bp.Px : (lane == 1 ? bp.Py : bp.Pz);
        const double Ac = lane == 0 ? A.x : (lane == 1 ? A.y : A.z);
        const double Bc = lane == 0 ? B.x : (lane == 1 ? B.y : B.z);
        warpmd::build_E1<LA, LB, T>(Eb + lane * WD::NEB, T(Pc - Ac), T(Pc - Bc), T(0.5 * bp.ip));
      }
      double wacc[MM::on ? MM::MT : 1][MM::on ? MM::NT : 1][2];
      if constexpr (MM::on) {
#pragma unroll
        for (int mt = 0; mt < MM::MT; ++mt)
#pragma unroll
          for (int nt = 0; nt < MM::NT; ++nt) wacc[mt][nt][0] = wacc[mt][nt][1] = 0.0;
      } else {
        for (int k = lane; k < WD::NW; k += 32) W[k] = T(0);
      }
      for (int ik = 0; ik < nk; ++ik) {
        const PrimPair kp = pkp[ik];
        __syncwarp();
        if (lane < 3) {
          const double Pc = lane == 0 ? kp.Px : (lane == 1 ? kp.Py : kp.Pz);
          const double Cc3 = lane == 0 ? C.x : (lane == 1 ? C.y : C.z);
          const double Dc = lane == 0 ? D.x : (lane == 1 ? D.y : D.z);
          warpmd::build_E1<LC, LD, T>(Ek + lane * WD::NEK, T(Pc - Cc3), T(Pc - Dc), T(0.5 * kp.ip));
        }
        const double pq = bp.p + kp.p;
        const double rpq = rsqrt(pq);
        const double rho = bp.p * kp.p * (rpq * rpq);
        const double X = bp.Px - kp.Px, Y = bp.Py - kp.Py, Z = bp.Pz - kp.Pz;
        double F[L + 1];
        boys_eval<L>(rho * (X * X + Y * Y + Z * Z), boys, F);
        double fac[L + 1];
        {
          double f = bp.Kp * kp.Kp * rpq;
          const double m2r = -2.0 * rho;
#pragma unroll
          for (int n = 0; n <= L; ++n) {
            fac[n] = f * F[n];
            f *= m2r;
          }
        }
        // R^{(n)}_{tuv}, n = L .. 0, ping-pong between Ra and Rb; level L in Ra when L even
        T *prev = (L % 2 == 0) ? Rb : Ra;
        T *cur = (L % 2 == 0) ? Ra : Rb;
        const T Xt = T(X), Yt = T(Y), Zt = T(Z);
        // level L: one entry
        if (lane == 0) cur[0] = T(fac[L]);
#pragma unroll
        for (int n = L - 1; n >= 0; --n) {
          T *t_ = prev;
          prev = cur;
          cur = t_;
          __syncwarp();
          const int cnt = warpmd::nherm(L - n);
          for (int h = lane; h < cnt; h += 32) {
            T val;
            if (h == 0) {
              val = T(fac[n]);
            } else {
              const int r = s_rec[h];
              const int dr = (r >> 20) & 3;
              const T pd = dr == 0 ? Xt : (dr == 1 ? Yt : Zt);
              val = pd * prev[r & 1023] + T(r >> 22) * prev[(r >> 10) & 1023];
            }
            cur[h] = val;
          }
        }
        __syncwarp();
        const T *R = cur;  // level 0
        if constexpr (MM::on) {
          // A[h][k] = R[h + k] gathered from shared memory, B[k][cd] = signed ket E product
          const int g = lane >> 2, tq = lane & 3;
          constexpr int NTQ = WD::Q + 1;
#pragma unroll
          for (int kt = 0; kt < MM::KT; ++kt) {
            const int k = kt * 4 + tq;
            double a[MM::MT];
#pragma unroll
            for (int mt = 0; mt < MM::MT; ++mt) {
              const int h = mt * 8 + g;
              a[mt] = (h < MM::HP && k < MM::HQ) ? (double)R[s_sum[h * MM::HQ + k]] : 0.0;
            }
            const int kc = k < MM::HQ ? s_h[k] : 0;
            const int kx = kc & 15, ky = (kc >> 4) & 15, kz = kc >> 8;
#pragma unroll
            for (int nt = 0; nt < MM::NT; ++nt) {
              const int c = nt * 8 + g;
              double b = 0.0;
              if (k < MM::HQ && c < NCCD) {
                const int cc = s_ccd[c];
                const int cx = cc & 15, cy = (cc >> 4) & 15, cz = (cc >> 8) & 15;
                const int dx = (cc >> 12) & 15, dy = (cc >> 16) & 15, dz = cc >> 20;
                if (kx <= cx + dx && ky <= cy + dy && kz <= cz + dz) {
                  b = (double)Ek[(cx * (LD + 1) + dx) * NTQ + kx] *
                      (double)Ek[WD::NEK + (cy * (LD + 1) + dy) * NTQ + ky] *
                      (double)Ek[2 * WD::NEK + (cz * (LD + 1) + dz) * NTQ + kz];
                  if ((kx + ky + kz) & 1) b = -b;
                }
              }
#pragma unroll
              for (int mt = 0; mt < MM::MT; ++mt) dmma_884(wacc[mt][nt], a[mt], b);
            }
          }
        } else if constexpr (MM::onS) {
          // the same product, with W read from and written back to shared memory for each
          // block of NTB column tiles (every element is owned by one lane throughout)
          const int g = lane >> 2, tq = lane & 3;
          constexpr int NTQ = WD::Q + 1;
          for (int n0 = 0; n0 < MM::NT; n0 += MM::NTB) {
            double wb[MM::MT][MM::NTB][2];
#pragma unroll
            for (int mt = 0; mt < MM::MT; ++mt)
#pragma unroll
              for (int j = 0; j < MM::NTB; ++j)
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                  const int h = mt * 8 + g, c = (n0 + j) * 8 + tq * 2 + i;
                  wb[mt][j][i] = (n0 + j < MM::NT && h < MM::HP && c < NCCD) ? (double)W[h * NCCD + c] : 0.0;
                }
#pragma unroll 1
            for (int kt = 0; kt < MM::KT; ++kt) {
              const int k = kt * 4 + tq;
              double a[MM::MT];
#pragma unroll
              for (int mt = 0; mt < MM::MT; ++mt) {
                const int h = mt * 8 + g;
                a[mt] = (h < MM::HP && k < MM::HQ) ? (double)R[s_sum[h * MM::HQ + k]] : 0.0;
              }
              const int kc = k < MM::HQ ? s_h[k] : 0;
              const int kx = kc & 15, ky = (kc >> 4) & 15, kz = kc >> 8;
#pragma unroll
              for (int j = 0; j < MM::NTB; ++j) {
                const int c = (n0 + j) * 8 + g;
                double b = 0.0;
                if (k < MM::HQ && n0 + j < MM::NT && c < NCCD) {
                  const int cc = s_ccd[c];
                  const int cx = cc & 15, cy = (cc >> 4) & 15, cz = (cc >> 8) & 15;
                  const int dx = (cc >> 12) & 15, dy = (cc >> 16) & 15, dz = cc >> 20;
                  if (kx <= cx + dx && ky <= cy + dy && kz <= cz + dz) {
                    b = (double)Ek[(cx * (LD + 1) + dx) * NTQ + kx] *
                        (double)Ek[WD::NEK + (cy * (LD + 1) + dy) * NTQ + ky] *
                        (double)Ek[2 * WD::NEK + (cz * (LD + 1) + dz) * NTQ + kz];
                    if ((kx + ky + kz) & 1) b = -b;
                  }
                }
#pragma unroll
                for (int mt = 0; mt < MM::MT; ++mt) dmma_884(wb[mt][j], a[mt], b);
              }
            }
#pragma unroll
            for (int mt = 0; mt < MM::MT; ++mt)
#pragma unroll
              for (int j = 0; j < MM::NTB; ++j)
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                  const int h = mt * 8 + g, c = (n0 + j) * 8 + tq * 2 + i;
                  if (n0 + j < MM::NT && h < MM::HP && c < NCCD) W[h * NCCD + c] = (T)wb[mt][j][i];
                }
          }
        } else
        // W[tuv][cd] += sum (-1)^(tau+nu+phi) E^cd R
        for (int e2 = lane; e2 < WD::NW; e2 += 32) {
          const int h = e2 / NCCD, c = e2 % NCCD;
          const int hc = s_h[h], cc = s_ccd[c];
          const int t = hc & 15, u = (hc >> 4) & 15, v = hc >> 8;
          const int cx = cc & 15, cy = (cc >> 4) & 15, cz = (cc >> 8) & 15;
          const int dx = (cc >> 12) & 15, dy = (cc >> 16) & 15, dz = cc >> 20;
          constexpr int NT = WD::Q + 1;
          const T *ex = Ek + (cx * (LD + 1) + dx) * NT;
          const T *ey = Ek + WD::NEK + (cy * (LD + 1) + dy) * NT;
          const T *ez = Ek + 2 * WD::NEK + (cz * (LD + 1) + dz) * NT;
          T s = T(0);
          for (int a1 = 0; a1 <= cx + dx; ++a1)
            for (int a2 = 0; a2 <= cy + dy; ++a2) {
              const T exy = ((a1 + a2) & 1 ? T(-1) : T(1)) * ex[a1] * ey[a2];
              for (int a3 = 0; a3 <= cz + dz; ++a3) {
                const T c3 = (a3 & 1) ? -ez[a3] : ez[a3];
                s += exy * c3 * R[warpmd::hidx(t + a1, u + a2, v + a3)];
              }
            }
          W[e2] += s;
        }
      }
      __syncwarp();
      if constexpr (MM::any) {
        const int g = lane >> 2, tq = lane & 3;
        constexpr int NTP = WD::P + 1;
        // W tiles to shared memory, then C[ab][cd] += EB[ab][h] W[h][cd] on the tensor cores
        if constexpr (MM::on) {
#pragma unroll
          for (int mt = 0; mt < MM::MT; ++mt)
#pragma unroll
            for (int nt = 0; nt < MM::NT; ++nt)
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int h = mt * 8 + g, c = nt * 8 + tq * 2 + i;
                if (h < MM::HP && c < NCCD) W[h * NCCD + c] = wacc[mt][nt][i];
              }
        }
        __syncwarp();
        for (int mtc = 0; mtc < MM::MTC; ++mtc) {
          const int abi = mtc * 8 + g;
          const int cab = abi < MM::NCAB ? s_cab[abi] : 0;
          const int ax = cab & 15, ay = (cab >> 4) & 15, az = (cab >> 8) & 15;
          const int bx = (cab >> 12) & 15, by = (cab >> 16) & 15, bz = cab >> 20;
          for (int nt = 0; nt < MM::NT; ++nt) {
            double cf[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int c = nt * 8 + tq * 2 + i;
              cf[i] = (abi < MM::NCAB && c < NCCD) ? (double)Cc[abi * NCCD + c] : 0.0;
            }
#pragma unroll
            for (int kt = 0; kt < MM::KTH; ++kt) {
              const int h = kt * 4 + tq;
              double a = 0.0;
              if (abi < MM::NCAB && h < MM::HP) {
                const int hc = s_h[h];
                const int t = hc & 15, u = (hc >> 4) & 15, v = hc >> 8;
                if (t <= ax + bx && u <= ay + by && v <= az + bz)
                  a = (double)Eb[(ax * (LB + 1) + bx) * NTP + t] *
                      (double)Eb[WD::NEB + (ay * (LB + 1) + by) * NTP + u] *
                      (double)Eb[2 * WD::NEB + (az * (LB + 1) + bz) * NTP + v];
              }
              const int hb = kt * 4 + tq, cb = nt * 8 + g;
              const double b = (hb < MM::HP && cb < NCCD) ? (double)W[hb * NCCD + cb] : 0.0;
              dmma_884(cf, a, b);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int c = nt * 8 + tq * 2 + i;
              if (abi < MM::NCAB && c < NCCD) Cc[abi * NCCD + c] = (T)cf[i];
            }
          }
        }
      } else
      // C[ab][cd] += sum_tuv E^ab_tuv W[tuv][cd]
      for (int e2 = lane; e2 < WD::NC; e2 += 32) {
        const int abi = e2 / NCCD, c = e2 % NCCD;
        const int cc = s_cab[abi];
        const int ax = cc & 15, ay = (cc >> 4) & 15, az = (cc >> 8) & 15;
        const int bx = (cc >> 12) & 15, by = (cc >> 16) & 15, bz = cc >> 20;
        constexpr int NT = WD::P + 1;
        const T *ex = Eb + (ax * (LB + 1) + bx) * NT;
        const T *ey = Eb + WD::NEB + (ay * (LB + 1) + by) * NT;
        const T *ez = Eb + 2 * WD::NEB + (az * (LB + 1) + bz) * NT;
        T s = T(0);
        for (int a1 = 0; a1 <= ax + bx; ++a1)
          for (int a2 = 0; a2 <= ay + by; ++a2) {
            const T exy = ex[a1] * ey[a2];
            for (int a3 = 0; a3 <= az + bz; ++a3) s += exy * ez[a3] * W[warpmd::hidx(a1, a2, a3) * NCCD + c];
          }
        Cc[e2] += s;
      }
    }
    __syncwarp();
    // Cartesian -> spherical on pure axes (L > 1), ping-pong Cc <-> W
    T *src = Cc, *dst = W;
    {
      int d[4] = {warpmd::ncart(LA), warpmd::ncart(LB), warpmd::ncart(LC), warpmd::ncart(LD)};
      const int ls[4] = {LA, LB, LC, LD};
#pragma unroll
      for (int ax = 0; ax < 4; ++ax) {
        if (ls[ax] < 2) continue;
        const double *Ct = ls[ax] == 2 ? kSph2 : kSph3;
        warpmd::sph_axis<T>(src, dst, d, ax, ls[ax], Ct, lane);
        d[ax] = 2 * ls[ax] + 1;
        T *t_ = src;
        src = dst;
        dst = t_;
        __syncwarp();
      }
    }
    const T *V = src;   // [a][b][c][d] in the reference basis
    constexpr int NA = WD::NSA, NB = WD::NSB, NC = WD::NSC, ND = WD::NSD;
    if (SCHWARZ) {
      double mx = 0.0;
      for (int k = lane; k < NA * NB; k += 32) mx = fmax(mx, fabs((double)V[k * (NA * NB) + k]));
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) Qout[q] = sqrt(mx);
      continue;
    }
    const double deg = (ab.x == ab.y ? 1.0 : 2.0) * (cdp.x == cdp.y ? 1.0 : 2.0) * (e.x == e.y ? 1.0 : 2.0);
    const int a0 = S.bf[ab.x], b0 = S.bf[ab.y], c0 = S.bf[cdp.x], d0 = S.bf[cdp.y];
    const int mol = S.mol[ab.x];
    // staged blocks: X(d,c) [NC*ND], X(b,a) [NA*NB], X(b,d), X(a,c), X(b,c), X(a,d)
    double *xdc = Xs, *xba = xdc + NC * ND, *xbd = xba + NA * NB, *xac = xbd + NB * ND;
    double *xbc = xac + NA * NC, *xad = xbc + NB * NC;
    for (int g = 0; g < dg.ng; ++g) {
      const double *Xv;
      double *G;
      size_t ld, n;
      mol_view(dg, g, mol, Xv, G, ld, n);
      const double *__restrict__ Xm = Xv;
      const double sJ = dg.sJ[g] * deg, sK = 0.5 * dg.sK[g] * deg;
      __syncwarp();
      for (int k = lane; k < NC * ND; k += 32) xdc[k] = __ldg(Xm + (d0 + k % ND) + (c0 + k / ND) * ld);
      for (int k = lane; k < NA * NB; k += 32) xba[k] = __ldg(Xm + (b0 + k % NB) + (a0 + k / NB) * ld);
      for (int k = lane; k < NB * ND; k += 32) xbd[k] = __ldg(Xm + (b0 + k / ND) + (d0 + k % ND) * ld);
      for (int k = lane; k < NA * NC; k += 32) xac[k] = __ldg(Xm + (a0 + k / NC) + (c0 + k % NC) * ld);
      for (int k = lane; k < NB * NC; k += 32) xbc[k] = __ldg(Xm + (b0 + k / NC) + (c0 + k % NC) * ld);
      for (int k = lane; k < NA * ND; k += 32) xad[k] = __ldg(Xm + (a0 + k / ND) + (d0 + k % ND) * ld);
      __syncwarp();
      // every update is written with the index that varies fastest across lanes as the
      // row (k_finalize symmetrises Gh), so a warp's atomics fall on consecutive addresses
      if (dg.sJ[g] != 0.0) {
        for (int k = lane; k < NA * NB; k += 32) {
          const int a = k / NB, b = k % NB;
          double s = 0.0;
          for (int cd = 0; cd < NC * ND; ++cd) s += xdc[cd] * V[k * NC * ND + cd];
          atomicAdd(G + (b0 + b) + (a0 + a) * n, sJ * s);
        }
        for (int k = lane; k < NC * ND; k += 32) {
          const int c = k / ND, d = k % ND;
          double s = 0.0;
          for (int ab2 = 0; ab2 < NA * NB; ++ab2) s += xba[ab2] * V[ab2 * NC * ND + k];
          atomicAdd(G + (d0 + d) + (c0 + c) * n, sJ * s);
        }
      }
      if (dg.sK[g] != 0.0) {
        for (int k = lane; k < NA * NC; k += 32) {   // G(a,c) += X(b,d) v
          const int a = k / NC, c = k % NC;
          double s = 0.0;
          for (int b = 0; b < NB; ++b)
            for (int d = 0; d < ND; ++d) s += xbd[b * ND + d] * V[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (c0 + c) + (a0 + a) * n, sK * s);
        }
        for (int k = lane; k < NB * ND; k += 32) {   // G(b,d) += X(a,c) v
          const int b = k / ND, d = k % ND;
          double s = 0.0;
          for (int a = 0; a < NA; ++a)
            for (int c = 0; c < NC; ++c) s += xac[a * NC + c] * V[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (d0 + d) + (b0 + b) * n, sK * s);
        }
        for (int k = lane; k < NA * ND; k += 32) {   // G(a,d) += X(b,c) v
          const int a = k / ND, d = k % ND;
          double s = 0.0;
          for (int b = 0; b < NB; ++b)
            for (int c = 0; c < NC; ++c) s += xbc[b * NC + c] * V[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (d0 + d) + (a0 + a) * n, sK * s);
        }
        for (int k = lane; k < NB * NC; k += 32) {   // G(b,c) += X(a,d) v
          const int b = k / NC, c = k % NC;
          double s = 0.0;
          for (int a = 0; a < NA; ++a)
            for (int d = 0; d < ND; ++d) s += xad[a * ND + d] * V[((a * NB + b) * NC + c) * ND + d];
          atomicAdd(G + (c0 + c) + (b0 + b) * n, sK * s);
        }
      }
    }
  }
}

template <int LA, int LB, int LC, int LD, typename T>
static size_t warp_smem_bytes() {
  using WD = warpmd::WarpDims<LA, LB, LC, LD>;
  constexpr int NBUF = (WD::NW > WD::NC) ? WD::NW : WD::NC;
  constexpr size_t WARP_BYTES = sizeof(double) * WD::NXS + sizeof(T) * (3 * WD::NEB + 3 * WD::NEK + 2 * WD::HL + 2 * NBUF);
  return 4 * ((WARP_BYTES + 15) / 16 * 16);
}

// AX += 0.5 (Gh + Gh^T), molecule blockIdx.z of the context
__global__ void k_finalize(const double *__restrict__ Gh0, Mols mols, double *__restrict__ AX0, int ldax) {
  __shared__ double tile[32][33];
  const int mol = blockIdx.z;
  const int n = mols.nbf[mol];
  if (!mols.active[mol] || (int)(blockIdx.x * 32) >= n || (int)(blockIdx.y * 32) >= n) return;
  const double *Gh = Gh0;
  double *AX = AX0;
  if (mols.nmol > 1) {
    Gh += mols.xoff[mol];
    AX += mols.xoff[mol];
    ldax = n;
  }
  int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int k = ty; k < 32; k += 8) {
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
  long long list_budget = 1LL << 32;   // quartets held in the list at once (8 B each: 32 GiB)
  int nsm = 148;                       // multiprocessors of the device
  // launch shapes per (precision, class) work list: persistent CTAs per SM and, for the
  // warp-cooperative classes, warps per CTA (0 = default); set by the autotuner
  int shape_cta[2 * CQG_NQC] = {0};
  int shape_wpb[2 * CQG_NQC] = {0};
  int autotune_pending = 0;
  long long graph_capacity = 0;        // > 0: sync-free contraction for CUDA-graph capture
  bool class_possible[CQG_NQC] = {false};
  // molecules of the context (a batch when nmol > 1)
  int nmol = 0, max_nsh = 0, max_nbf = 0;
  long long packed = 0, Mtotal = 0, nallpairs = 0;
  std::vector<int> hshmol, m_shoff, m_nsh, m_nbf;
  std::vector<long long> m_xoff, m_Moff;
  std::vector<unsigned char> h_active;
  DevBuf<int> d_shmol, d_mshoff, d_mnsh, d_mnbf, d_molbk;
  DevBuf<long long> d_mxoff, d_mMoff;
  DevBuf<unsigned char> d_active;
  // basis
  int nshell = 0, nbf = 0, maxl = 0;
  std::vector<int> hL, hbf, hsz, hnprim, hpoff;
  std::vector<double> halpha, hcoef, hcent;
  std::vector<double> Qmat;  // nshell x nshell
  // pairs, by class
  int pc_beg[CQG_NPC + 1] = {0};
  int bucket_beg[CQG_NPC][CQG_NBUCKET + 1];
  std::vector<int2> pair_sh;
  std::vector<double> pair_Q;
  DevBuf<double3> d_center;
  DevBuf<int> d_bf, d_sz;
  DevBuf<int2> d_pair_sh;
  DevBuf<double> d_pair_Q;
  DevBuf<int> d_pair_poff, d_pair_np, d_pair_kk;
  DevBuf<int> d_shL, d_shnp, d_shpoff;
  DevBuf<double> d_alpha, d_coef;
  DevBuf<int2> d_allpairs;
  DevBuf<double> d_oe;       // host-mode staging of S, T, V
  DevBuf<double> d_charges;  // Z then R (3 per charge)
  DevBuf<unsigned long long> d_blkacc;
  int launches = 0;
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
  DevBuf<double> d_G, d_X, d_AX, d_Gscratch;
  BlockTable bt;
  int ntask = 0;
  cudaEvent_t ev[4 + 2 * 55];
  bool events = false;
  cqg_stats stats;
  double *oe_table = nullptr;   // device address of the fixed charge table (cqg_one_e_noalloc)
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

static Pairs make_pairs(cqg_ctx *ctx);
static Shells make_shells(cqg_ctx *ctx);

// classes evaluated by the warp-cooperative kernel (same rule as gen_eri.WARP_CLASSES)
__host__ __device__ constexpr bool is_warp_class(int la, int lb, int lc, int ld) {
  return ncart_c(la) * ncart_c(lb) * ncart_c(lc) * ncart_c(ld) > 150 || la + lb + lc + ld >= 6;
}

template <int LA, int LB, int LC, int LD, bool SCHWARZ, typename T>
static cudaError_t launch_warp(cqg_ctx *ctx, int blk, long long n, long long sbeg, long long send, cudaStream_t st,
                               const DigestGroups &dg, double *Q) {
  if (n == 0) return cudaSuccess;   // n < 0: count unknown on the host (graph mode)
  // the attribute belongs to the kernel on each device: set it once per device
  static bool attr_set[64] = {};
  const size_t per_warp = warp_smem_bytes<LA, LB, LC, LD, T>() / 4;
  const int wpb_max = (int)std::max<size_t>(1, std::min<size_t>(4, (200u * 1024u) / per_warp));
  const int dev_slot = (ctx->device >= 0 && ctx->device < 64) ? ctx->device : 0;
  if (!attr_set[dev_slot]) {
    cudaError_t e = cudaFuncSetAttribute(k_eri_jk_warp<LA, LB, LC, LD, SCHWARZ, T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(per_warp * wpb_max));
    if (e != cudaSuccess) return e;
    attr_set[dev_slot] = true;
  }
  int wpb = wpb_max, cta = 16;
  if (!SCHWARZ && ctx->shape_wpb[blk] > 0) wpb = std::min(wpb_max, ctx->shape_wpb[blk]);
  if (!SCHWARZ && ctx->shape_cta[blk] > 0) cta = ctx->shape_cta[blk];
  const size_t smem = per_warp * wpb;
  const long long cap = (long long)ctx->nsm * cta;
  const int blocks = (int)(n > 0 ? std::min<long long>((n + wpb - 1) / wpb, cap) : cap);
  k_eri_jk_warp<LA, LB, LC, LD, SCHWARZ, T><<<blocks, 32 * wpb, smem, st>>>(ctx->d_qlist.p, ctx->d_range.p, blk, sbeg,
                                                                       send, make_pairs(ctx), make_shells(ctx),
                                                                       ctx->d_boys.p, dg, Q);
  return cudaGetLastError();
}

template <int LA, int LB>
static cudaError_t launch_schwarz(cqg_ctx *ctx, Pairs P, Shells S, int beg, int end, double *Q) {
  int n = end - beg;
  if (n <= 0) return cudaSuccess;
  if constexpr (is_warp_class(LA, LB, LA, LB)) {
    DigestGroups dg;
    memset(&dg, 0, sizeof(dg));
    return launch_warp<LA, LB, LA, LB, true, double>(ctx, 0, n, beg, end, 0, dg, Q);
  } else {
    k_schwarz<LA, LB><<<(n + 127) / 128, 128>>>(P, S, ctx->d_boys.p, beg, end, Q);
    return cudaGetLastError();
  }
}

static Pairs make_pairs(cqg_ctx *ctx) {
  Pairs P;
  P.sh = ctx->d_pair_sh.p;
  P.Q = ctx->d_pair_Q.p;
  P.poff = ctx->d_pair_poff.p;
  P.np = ctx->d_pair_np.p;
  P.kk = ctx->d_pair_kk.p;
  P.prim = ctx->d_prim.p;
  return P;
}
static Shells make_shells(cqg_ctx *ctx) {
  Shells S;
  S.center = ctx->d_center.p;
  S.bf = ctx->d_bf.p;
  S.mol = ctx->d_shmol.p;
  return S;
}
static Mols make_mols(cqg_ctx *ctx) {
  Mols M;
  M.nmol = ctx->nmol;
  M.shoff = ctx->d_mshoff.p;
  M.nsh = ctx->d_mnsh.p;
  M.Moff = ctx->d_mMoff.p;
  M.xoff = ctx->d_mxoff.p;
  M.nbf = ctx->d_mnbf.p;
  M.active = ctx->d_active.p;
  M.molbk = ctx->d_molbk.p;
  return M;
}

// Primitive pairs of shell pair (a, b); prim_thresh = 0 keeps all of them, otherwise a
// pair whose s-type bound sqrt((ij|ij)) (with a (1+|AB|)^(la+lb) allowance) is below
// prim_thresh is dropped.
static void pair_prims(const cqg_ctx *ctx, int a, int b, double prim_thresh, std::vector<PrimPair> &out) {
  const double pi = 3.14159265358979323846;
  const double s2pi52 = std::sqrt(2.0 * std::pow(pi, 2.5));
  const double *A = &ctx->hcent[3 * a], *B = &ctx->hcent[3 * b];
  double AB2 = 0;
  for (int x = 0; x < 3; ++x) AB2 += (A[x] - B[x]) * (A[x] - B[x]);
  const double ABn = std::sqrt(AB2);
  for (int ia = 0; ia < ctx->hnprim[a]; ++ia)
    for (int ib = 0; ib < ctx->hnprim[b]; ++ib) {
      double al = ctx->halpha[ctx->hpoff[a] + ia], be = ctx->halpha[ctx->hpoff[b] + ib];
      double ca = ctx->hcoef[ctx->hpoff[a] + ia], cb = ctx->hcoef[ctx->hpoff[b] + ib];
      double p = al + be;
      double K = ca * cb * std::exp(-al * be / p * AB2);
      if (prim_thresh > 0) {
        double bound = std::fabs(K) * s2pi52 / (p * std::pow(2.0 * p, 0.25)) * std::pow(1.0 + ABn, ctx->hL[a] + ctx->hL[b]);
        if (bound < prim_thresh) continue;
      }
      PrimPair pp;
      pp.p = p;
      pp.ip = 1.0 / p;
      pp.Kp = s2pi52 * K / p;
      pp.Px = (al * A[0] + be * B[0]) / p;
      pp.Py = (al * A[1] + be * B[1]) / p;
      pp.Pz = (al * A[2] + be * B[2]) / p;
      out.push_back(pp);
    }
}

// primitive-count bucket of a shell pair: warps of the ERI kernels see kets of one bucket
static inline int prim_bucket(int np) {
  static const int upper[CQG_NBUCKET - 1] = {1, 2, 3, 4, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64};
  for (int b = 0; b < CQG_NBUCKET - 1; ++b)
    if (np <= upper[b]) return b;
  return CQG_NBUCKET - 1;
}

// build primitive-pair data for the current pair ordering and upload all pair arrays
static cqg_status upload_pairs(cqg_ctx *ctx, double prim_thresh) {
  size_t np = ctx->pair_sh.size();
  std::vector<int> poff(np), npr(np), kk(np);
  std::vector<PrimPair> prim;
  prim.reserve(np * 4);
  for (size_t i = 0; i < np; ++i) {
    int a = ctx->pair_sh[i].x, b = ctx->pair_sh[i].y;
    poff[i] = (int)prim.size();
    kk[i] = ctx->hnprim[a] * ctx->hnprim[b];
    pair_prims(ctx, a, b, prim_thresh, prim);
    npr[i] = (int)prim.size() - poff[i];
  }
  ctx->prim_pairs_total = (long long)prim.size();
  ctx->pair_np_host = npr;
  if (ctx->d_pair_sh.reserve(np) || ctx->d_pair_Q.reserve(np) || ctx->d_pair_poff.reserve(np) ||
      ctx->d_pair_np.reserve(np) || ctx->d_pair_kk.reserve(np) || ctx->d_prim.reserve(prim.size())) {
    ctx->err = "device allocation for pair data failed";
    return CQG_ERR_OOM;
  }
  CUCHK(cudaMemcpy(ctx->d_pair_sh.p, ctx->pair_sh.data(), np * sizeof(int2), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_Q.p, ctx->pair_Q.data(), np * sizeof(double), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_poff.p, poff.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_np.p, npr.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_pair_kk.p, kk.data(), np * sizeof(int), cudaMemcpyHostToDevice));
  if (!prim.empty())
    CUCHK(cudaMemcpy(ctx->d_prim.p, prim.data(), prim.size() * sizeof(PrimPair), cudaMemcpyHostToDevice));
  return CQG_OK;
}

typedef cudaError_t (*eri_launcher)(cqg_ctx *, int blk, long long n, cudaStream_t st, const DigestGroups &dg);

template <int LA, int LB, int LC, int LD, typename T>
static cudaError_t launch_eri(cqg_ctx *ctx, int blk, long long n, cudaStream_t st, const DigestGroups &dg) {
  if (n == 0) return cudaSuccess;   // n < 0: count unknown on the host (graph mode)
  if constexpr (is_warp_class(LA, LB, LC, LD)) {
    return launch_warp<LA, LB, LC, LD, false, T>(ctx, blk, n, 0, 0, st, dg, nullptr);
  } else {
    const int cta = ctx->shape_cta[blk] > 0 ? ctx->shape_cta[blk] : 12;
    const long long cap = (long long)ctx->nsm * cta;
    long long nb = n > 0 ? std::min<long long>((n + kEriThreads - 1) / kEriThreads, cap) : cap;
    k_eri_jk<LA, LB, LC, LD, T><<<(unsigned)nb, kEriThreads, 0, st>>>(ctx->d_qlist.p, ctx->d_range.p, blk,
                                                                   make_pairs(ctx), make_shells(ctx), ctx->d_boys.p,
                                                                   dg);
    return cudaGetLastError();
  }
}

#define QC(a, b, c, d, T) &launch_eri<a, b, c, d, T>
static const eri_launcher kEriLaunch[CQG_NQC] = CQG_CLASS_LIST(QC, double);
static const eri_launcher kEriLaunch32[CQG_NQC] = CQG_CLASS_LIST(QC, float);
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
  std::vector<double> tab(BOYS_TABLE_SIZE);
  for (int i = 0; i < BOYS_NT; ++i) host_boys_row(BOYS_NORD - 1, (long double)i / 10.0L, &tab[i * BOYS_NORD]);
  for (int i = 0; i < BOYS_NT; ++i) tab[BOYS_NT * BOYS_NORD + i] = (double)expl(-(long double)i / 10.0L);
  if (ctx->d_boys.reserve(tab.size()) != cudaSuccess ||
      cudaMemcpy(ctx->d_boys.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete ctx;
    return CQG_ERR_CUDA;
  }
  for (int i = 0; i < 4 + 2 * 55; ++i) cudaEventCreate(&ctx->ev[i]);
  ctx->events = true;
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
  *out = ctx;
  return CQG_OK;
}

cqg_status cqg_destroy(cqg_ctx *ctx) {
  if (!ctx) return CQG_OK;
  cudaSetDevice(ctx->device);
  ctx->d_center.release(); ctx->d_bf.release(); ctx->d_sz.release();
  ctx->d_pair_sh.release(); ctx->d_pair_Q.release(); ctx->d_pair_poff.release(); ctx->d_pair_np.release();
  ctx->d_pair_kk.release(); ctx->d_blkacc.release();
  ctx->d_shL.release(); ctx->d_shnp.release(); ctx->d_shpoff.release(); ctx->d_alpha.release();
  ctx->d_coef.release(); ctx->d_allpairs.release(); ctx->d_oe.release(); ctx->d_charges.release();
  ctx->d_shmol.release(); ctx->d_mshoff.release(); ctx->d_mnsh.release(); ctx->d_mnbf.release();
  ctx->d_molbk.release(); ctx->d_mxoff.release(); ctx->d_mMoff.release(); ctx->d_active.release();
  ctx->d_prim.release(); ctx->d_boys.release();
  ctx->d_M.release(); ctx->d_Mmax.release(); ctx->d_flags.release();
  ctx->d_cnt.release(); ctx->d_off.release(); ctx->d_range.release(); ctx->d_scan_tmp.release();
  ctx->d_qlist.release(); ctx->d_G.release(); ctx->d_X.release(); ctx->d_AX.release(); ctx->d_Gscratch.release();
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

cqg_status cqg_set_list_budget(cqg_ctx *ctx, long long quartets) {
  if (!ctx || quartets < 1) return CQG_ERR_BAD_ARG;
  ctx->list_budget = quartets;
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

cqg_status cqg_set_basis_batch(cqg_ctx *ctx, int nmol, const int *nshell_per_mol, const int *L, const int *pure,
                               const int *nprim, const double *alpha, const double *coef, const double *centers) {
  if (!ctx || nmol <= 0 || !nshell_per_mol || !L || !pure || !nprim || !alpha || !coef || !centers)
    return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  int nshell = 0;
  for (int m = 0; m < nmol; ++m) {
    if (nshell_per_mol[m] <= 0) {
      ctx->err = "molecule without shells";
      return CQG_ERR_BAD_ARG;
    }
    nshell += nshell_per_mol[m];
  }
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
  ctx->nmol = nmol;
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
  ctx->hshmol.resize(nshell);
  ctx->m_shoff.resize(nmol);
  ctx->m_nsh.resize(nmol);
  ctx->m_nbf.resize(nmol);
  ctx->m_xoff.resize(nmol);
  ctx->m_Moff.resize(nmol);
  {
    int p = 0, s = 0;
    long long xo = 0, mo = 0;
    ctx->max_nsh = 0;
    ctx->max_nbf = 0;
    for (int m = 0; m < nmol; ++m) {
      ctx->m_shoff[m] = s;
      ctx->m_nsh[m] = nshell_per_mol[m];
      int f = 0;
      for (int k = 0; k < nshell_per_mol[m]; ++k, ++s) {
        ctx->hbf[s] = f;
        ctx->hsz[s] = nfun(L[s]);
        f += ctx->hsz[s];
        ctx->hpoff[s] = p;
        p += nprim[s];
        ctx->hshmol[s] = m;
      }
      ctx->m_nbf[m] = f;
      ctx->m_xoff[m] = xo;
      ctx->m_Moff[m] = mo;
      xo += (long long)f * f;
      mo += (long long)nshell_per_mol[m] * nshell_per_mol[m];
      ctx->max_nsh = std::max(ctx->max_nsh, nshell_per_mol[m]);
      ctx->max_nbf = std::max(ctx->max_nbf, f);
    }
    ctx->packed = xo;
    ctx->Mtotal = mo;
  }
  ctx->nbf = ctx->m_nbf[0];
  // shells and molecule layout to device
  std::vector<double3> c3(nshell);
  for (int s = 0; s < nshell; ++s) c3[s] = make_double3(centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]);
  if (ctx->d_center.reserve(nshell) || ctx->d_bf.reserve(nshell) || ctx->d_sz.reserve(nshell) ||
      ctx->d_shmol.reserve(nshell) || ctx->d_mshoff.reserve(nmol) || ctx->d_mnsh.reserve(nmol) ||
      ctx->d_mnbf.reserve(nmol) || ctx->d_mxoff.reserve(nmol) || ctx->d_mMoff.reserve(nmol) ||
      ctx->d_active.reserve(nmol))
    return CQG_ERR_OOM;
  CUCHK(cudaMemcpy(ctx->d_center.p, c3.data(), nshell * sizeof(double3), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_bf.p, ctx->hbf.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_sz.p, ctx->hsz.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_shmol.p, ctx->hshmol.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mshoff.p, ctx->m_shoff.data(), nmol * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mnsh.p, ctx->m_nsh.data(), nmol * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mnbf.p, ctx->m_nbf.data(), nmol * sizeof(int), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mxoff.p, ctx->m_xoff.data(), nmol * sizeof(long long), cudaMemcpyHostToDevice));
  CUCHK(cudaMemcpy(ctx->d_mMoff.p, ctx->m_Moff.data(), nmol * sizeof(long long), cudaMemcpyHostToDevice));
  ctx->h_active.assign(nmol, 1);
  CUCHK(cudaMemcpy(ctx->d_active.p, ctx->h_active.data(), nmol, cudaMemcpyHostToDevice));
  // raw shells (one-electron integrals) and the list of all pairs a >= b within each molecule
  {
    std::vector<int2> allp;
    for (int m = 0; m < nmol; ++m)
      for (int a = ctx->m_shoff[m]; a < ctx->m_shoff[m] + ctx->m_nsh[m]; ++a)
        for (int b = ctx->m_shoff[m]; b <= a; ++b) allp.push_back(make_int2(a, b));
    ctx->nallpairs = (long long)allp.size();
    if (ctx->d_shL.reserve(nshell) || ctx->d_shnp.reserve(nshell) || ctx->d_shpoff.reserve(nshell) ||
        ctx->d_alpha.reserve(tot) || ctx->d_coef.reserve(tot) || ctx->d_allpairs.reserve(allp.size()))
      return CQG_ERR_OOM;
    CUCHK(cudaMemcpy(ctx->d_shL.p, L, nshell * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_shnp.p, nprim, nshell * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_shpoff.p, ctx->hpoff.data(), nshell * sizeof(int), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_alpha.p, alpha, tot * sizeof(double), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_coef.p, coef, tot * sizeof(double), cudaMemcpyHostToDevice));
    CUCHK(cudaMemcpy(ctx->d_allpairs.p, allp.data(), allp.size() * sizeof(int2), cudaMemcpyHostToDevice));
  }
  // pairs within each molecule, by class, internal orientation L_a >= L_b (a >= b when equal L)
  std::vector<std::vector<int2>> bycls(CQG_NPC);
  for (int m = 0; m < nmol; ++m)
    for (int a = ctx->m_shoff[m]; a < ctx->m_shoff[m] + ctx->m_nsh[m]; ++a)
      for (int b = ctx->m_shoff[m]; b <= a; ++b) {
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
  e = e ? e : launch_schwarz<3, 0>(ctx, P, S, ctx->pc_beg[6], ctx->pc_beg[7], dQ);
  e = e ? e : launch_schwarz<3, 1>(ctx, P, S, ctx->pc_beg[7], ctx->pc_beg[8], dQ);
  e = e ? e : launch_schwarz<3, 2>(ctx, P, S, ctx->pc_beg[8], ctx->pc_beg[9], dQ);
  e = e ? e : launch_schwarz<3, 3>(ctx, P, S, ctx->pc_beg[9], ctx->pc_beg[10], dQ);
  if (e != cudaSuccess) {
    ctx->err = std::string("schwarz kernels: ") + cudaGetErrorString(e);
    return CQG_ERR_CUDA;
  }
  CUCHK(cudaDeviceSynchronize());
  CUCHK(cudaMemcpy(ctx->pair_Q.data(), dQ, ctx->pair_Q.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (nmol == 1) {
    ctx->Qmat.assign((size_t)nshell * nshell, 0.0);
    for (size_t i = 0; i < ctx->pair_sh.size(); ++i) {
      int a = ctx->pair_sh[i].x, b = ctx->pair_sh[i].y;
      ctx->Qmat[a + (size_t)b * nshell] = ctx->pair_Q[i];
      ctx->Qmat[b + (size_t)a * nshell] = ctx->pair_Q[i];
    }
  } else {
    ctx->Qmat.clear();
  }
  // sort each class by (molecule, primitive-count bucket, Q descending), stable, and
  // rebuild with primitive-pair screening; per (molecule, class) bucket starts -> molbk
  std::vector<int> npscr(ctx->pair_sh.size());
  {
    std::vector<PrimPair> tmp;
    for (size_t i = 0; i < ctx->pair_sh.size(); ++i) {
      tmp.clear();
      pair_prims(ctx, ctx->pair_sh[i].x, ctx->pair_sh[i].y, 1e-24, tmp);
      npscr[i] = (int)tmp.size();
    }
  }
  const int NB1 = CQG_NBUCKET + 1;
  std::vector<int> molbk((size_t)nmol * CQG_NPC * NB1, 0);
  for (int c = 0; c < CQG_NPC; ++c) {
    int b0 = ctx->pc_beg[c], b1 = ctx->pc_beg[c + 1];
    std::vector<int> idx(b1 - b0);
    std::iota(idx.begin(), idx.end(), b0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
      int mx = ctx->hshmol[ctx->pair_sh[x].x], my = ctx->hshmol[ctx->pair_sh[y].x];
      if (mx != my) return mx < my;
      int bx = prim_bucket(npscr[x]), by = prim_bucket(npscr[y]);
      if (bx != by) return bx < by;
      return ctx->pair_Q[x] > ctx->pair_Q[y];
    });
    // bucket starts per molecule: first index of (m, bk); empty buckets start where the next begins
    std::vector<int> first((size_t)nmol * NB1, -1);
    for (int k = 0; k < (int)idx.size(); ++k) {
      const int m = ctx->hshmol[ctx->pair_sh[idx[k]].x], bk = prim_bucket(npscr[idx[k]]);
      if (first[(size_t)m * NB1 + bk] < 0) first[(size_t)m * NB1 + bk] = b0 + k;
    }
    int next = b1;
    for (int m = nmol - 1; m >= 0; --m) {
      int *row = &molbk[((size_t)m * CQG_NPC + c) * NB1];
      row[CQG_NBUCKET] = next;
      for (int bk = CQG_NBUCKET - 1; bk >= 0; --bk) {
        const int f = first[(size_t)m * NB1 + bk];
        row[bk] = f >= 0 ? f : row[bk + 1];
      }
      next = row[0];
    }
    for (int bk = 0; bk <= CQG_NBUCKET; ++bk) ctx->bucket_beg[c][bk] = molbk[(size_t)c * NB1 + bk];
    std::vector<int2> sh2;
    std::vector<double> q2;
    for (int i : idx) {
      sh2.push_back(ctx->pair_sh[i]);
      q2.push_back(ctx->pair_Q[i]);
    }
    std::copy(sh2.begin(), sh2.end(), ctx->pair_sh.begin() + b0);
    std::copy(q2.begin(), q2.end(), ctx->pair_Q.begin() + b0);
  }
  if (ctx->d_molbk.reserve(molbk.size())) return CQG_ERR_OOM;
  CUCHK(cudaMemcpy(ctx->d_molbk.p, molbk.data(), molbk.size() * sizeof(int), cudaMemcpyHostToDevice));
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
    bt.ket_class[k] = j;
    bt.diag[k] = (i == j);
    task += ctx->pc_beg[i + 1] - ctx->pc_beg[i];
  }
  bt.task_beg[CQG_NQC] = task;
  bt.nblk = CQG_NQC;
  ctx->ntask = task;
  for (int k = 0; k < CQG_NQC; ++k) {
    int i, j;
    qclass_split(k, i, j);
    ctx->class_possible[k] = ctx->pc_beg[i + 1] > ctx->pc_beg[i] && ctx->pc_beg[j + 1] > ctx->pc_beg[j];
  }
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (long long *)nullptr, (long long *)nullptr, std::max(2 * task, 1));
  if (ctx->d_cnt.reserve(2 * task + 1) || ctx->d_off.reserve(2 * task + 1) || ctx->d_range.reserve(4 * CQG_NQC) ||
      ctx->d_scan_tmp.reserve(scan_bytes + 16) || ctx->d_M.reserve(2 * (size_t)std::max(ctx->Mtotal, 1LL)) ||
      ctx->d_Mmax.reserve(1) || ctx->d_flags.reserve(4) || ctx->d_blkacc.reserve(4 * CQG_NQC))
    return CQG_ERR_OOM;
  return CQG_OK;
}

cqg_status cqg_set_basis(cqg_ctx *ctx, int nshell, const int *L, const int *pure, const int *nprim,
                         const double *alpha, const double *coef, const double *centers) {
  return cqg_set_basis_batch(ctx, 1, &nshell, L, pure, nprim, alpha, coef, centers);
}

cqg_status cqg_get_schwarz(cqg_ctx *ctx, double *Q) {
  if (!ctx || !Q) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  memcpy(Q, ctx->Qmat.data(), ctx->Qmat.size() * sizeof(double));
  return CQG_OK;
}

// Launch-shape autotuner: for every (precision, class) list with work, time each candidate
// shape (persistent CTAs per SM; warps per CTA for the warp-cooperative classes) with the
// digest pointed at scratch accumulators, and keep the fastest.
static cqg_status autotune_shapes(cqg_ctx *ctx, const long long *crange, cudaStream_t st, const DigestGroups &dg) {
  DigestGroups scratch = dg;
  size_t per = 0;
  for (int g = 0; g < dg.ng; ++g) per = std::max<size_t>(per, 1);
  const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)ctx->nbf * ctx->nbf;
  if (ctx->d_Gscratch.reserve(gsize) != cudaSuccess) return CQG_ERR_OOM;
  for (int g = 0; g < dg.ng; ++g) scratch.G[g] = ctx->d_Gscratch.p;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int vb = 0; vb < 2 * CQG_NQC; ++vb) {
    const long long n = crange[2 * vb + 1] - crange[2 * vb];
    if (n <= 0) continue;
    const int k = vb % CQG_NQC;
    int i, j;
    qclass_split(k, i, j);
    const bool warp = is_warp_class(kPairClass[i][0], kPairClass[i][1], kPairClass[j][0], kPairClass[j][1]);
    std::vector<std::pair<int, int>> cand;   // (cta per SM, warps per CTA)
    if (warp) {
      for (int w : {1, 2, 4})
        for (int c : {8, 16, 32}) cand.push_back({c, w});
    } else {
      for (int c : {4, 8, 12, 16, 24}) cand.push_back({c, 0});
    }
    // Long lists are timed on their first quarter (at least 2^20 quartets), after one
    // untimed run, one run per candidate; short lists in full, best of two runs.  The
    // kernels read their range from d_range, so the sample range is written there and the
    // full range put back afterwards.
    const long long m = n > (1ll << 20) ? std::max<long long>(1ll << 20, n / 4) : n;
    const int reps = m < n ? 1 : 2;
    if (m < n) {
      const long long sub[2] = {crange[2 * vb], crange[2 * vb] + m};
      CUCHK(cudaMemcpyAsync(ctx->d_range.p + 2 * vb, sub, sizeof(sub), cudaMemcpyHostToDevice, st));
    }
    float best = 1e30f;
    std::pair<int, int> pick = cand[0];
    for (int ci = (m < n ? -1 : 0); ci < (int)cand.size(); ++ci) {
      const std::pair<int, int> cw = cand[ci < 0 ? 0 : ci];
      ctx->shape_cta[vb] = cw.first;
      ctx->shape_wpb[vb] = cw.second;
      float tbest = 1e30f;
      for (int rep = 0; rep < (ci < 0 ? 1 : reps); ++rep) {
        cudaEventRecord(e0, st);
        cudaError_t e = (vb < CQG_NQC ? kEriLaunch[k] : kEriLaunch32[k])(ctx, vb, m, st, scratch);
        cudaEventRecord(e1, st);
        if (e != cudaSuccess) {
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
          ctx->err = std::string("autotune launch: ") + cudaGetErrorString(e);
          return CQG_ERR_CUDA;
        }
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        tbest = std::min(tbest, ms);
      }
      if (ci >= 0 && tbest < best) {
        best = tbest;
        pick = cw;
      }
    }
    if (m < n) CUCHK(cudaMemcpyAsync(ctx->d_range.p + 2 * vb, crange + 2 * vb, 2 * sizeof(long long),
                                     cudaMemcpyHostToDevice, st));
    ctx->shape_cta[vb] = pick.first;
    ctx->shape_wpb[vb] = pick.second;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return CQG_OK;
}

// Sync-free contraction for CUDA-graph capture: the quartet list has a fixed capacity,
// every class kernel reads its range from device memory and runs a persistent grid, and
// nothing is read back.  Overflow of the capacity and invalid inputs are reported through
// device flags (cqg_graph_status).
static cqg_status contract_graph(cqg_ctx *ctx, int ngroups, const double *const *Xg, double *const *AXg,
                                 const double *sJ, const double *sK, int nx_all, const double *const *Xall, int ldx,
                                 int ldax, cudaStream_t st) {
  const Mols mols = make_mols(ctx);
  const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)ctx->nbf * ctx->nbf;
  if ((size_t)ngroups * gsize > ctx->d_G.n || (size_t)ctx->graph_capacity > ctx->d_qlist.n) {
    ctx->err = "graph mode: buffers were not reserved for this call (cqg_set_graph_mode)";
    return CQG_ERR_STATE;
  }
  XList xl;
  xl.n = nx_all;
  for (int i = 0; i < nx_all; ++i) xl.X[i] = Xall[i];
  const double cut32 = ctx->policy == CQG_PREC_MIXED ? ctx->fp32_cutoff : 0.0;
  CUCHK(cudaMemsetAsync(ctx->d_flags.p, 0, 4 * sizeof(int), st));
  CUCHK(cudaMemsetAsync(ctx->d_Mmax.p, 0, sizeof(double), st));
  CUCHK(cudaMemsetAsync(ctx->d_blkacc.p, 0, 4 * CQG_NQC * sizeof(unsigned long long), st));
  CUCHK(cudaMemsetAsync(ctx->d_G.p, 0, (size_t)ngroups * gsize * sizeof(double), st));
  {
    dim3 g((ctx->max_nsh + 127) / 128, ctx->max_nsh, ctx->nmol);
    k_blocknorm<<<g, 128, 0, st>>>(xl, ldx, mols, ctx->d_bf.p, ctx->d_sz.p, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_flags.p, 1e-12);
    const long long nn = ctx->Mtotal;
    k_maxreduce<<<(int)std::min<long long>((nn + 255) / 256, 1184), 256, 0, st>>>(ctx->d_M.p, nn, ctx->d_Mmax.p);
  }
  Pairs P = make_pairs(ctx);
  const int nb = (ctx->ntask + 7) / 8;
  k_quartets<false><<<nb, 256, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                         ctx->thresh, cut32, ctx->d_cnt.p, nullptr, nullptr, ctx->d_blkacc.p, 0, 0, 0,
                                         0);
  size_t scan_bytes = ctx->d_scan_tmp.n;
  CUCHK(cub::DeviceScan::ExclusiveSum(ctx->d_scan_tmp.p, scan_bytes, ctx->d_cnt.p, ctx->d_off.p, 2 * ctx->ntask, st));
  k_block_ranges<<<1, 128, 0, st>>>(ctx->bt, ctx->ntask, ctx->d_cnt.p, ctx->d_off.p, ctx->d_range.p,
                                    ctx->graph_capacity, ctx->d_flags.p);
  k_quartets<true><<<nb, 256, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                        ctx->thresh, cut32, nullptr, ctx->d_off.p, ctx->d_qlist.p, nullptr, 0,
                                        2LL * ctx->ntask, 0, ctx->graph_capacity);
  CUCHK(cudaGetLastError());
  DigestGroups dg;
  memset(&dg, 0, sizeof(dg));
  dg.ng = ngroups;
  dg.ldx = ldx;
  dg.batch = ctx->nmol > 1;
  dg.xoff = ctx->d_mxoff.p;
  dg.nbf = ctx->d_mnbf.p;
  for (int g = 0; g < ngroups; ++g) {
    dg.X[g] = Xg[g];
    dg.G[g] = ctx->d_G.p + (size_t)g * gsize;
    dg.sJ[g] = sJ[g];
    dg.sK[g] = sK[g];
  }
  int launches = 6;
  for (int k = 0; k < CQG_NQC; ++k) {
    if (!ctx->class_possible[k]) continue;
    cudaError_t e = kEriLaunch[k](ctx, k, -1, st, dg);
    ++launches;
    if (e == cudaSuccess && ctx->policy == CQG_PREC_MIXED) {
      e = kEriLaunch32[k](ctx, CQG_NQC + k, -1, st, dg);
      ++launches;
    }
    if (e != cudaSuccess) {
      ctx->err = std::string("eri kernel ") + cqg_class_name(k) + ": " + cudaGetErrorString(e);
      return CQG_ERR_CUDA;
    }
  }
  for (int g = 0; g < ngroups; ++g) {
    dim3 grid((ctx->max_nbf + 31) / 32, (ctx->max_nbf + 31) / 32, ctx->nmol), blk(32, 8);
    k_finalize<<<grid, blk, 0, st>>>(dg.G[g], mols, AXg[g], ldax);
    ++launches;
  }
  CUCHK(cudaGetLastError());
  ctx->launches = launches;
  ctx->stats.launches = launches;
  return CQG_OK;
}

static cqg_status contract_device(cqg_ctx *ctx, int ngroups, const double *const *Xg, double *const *AXg,
                                  const double *sJ, const double *sK, int nx_all, const double *const *Xall,
                                  int ldx, int ldax, cudaStream_t st) {
  const int n = ctx->nbf;
  const Mols mols = make_mols(ctx);
  // Gh of every molecule: n x n for one molecule, packed per molecule for a batch
  const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)n * n;
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[0], st));
  // 1. block norms + checks
  XList xl;
  xl.n = nx_all;
  for (int i = 0; i < nx_all; ++i) xl.X[i] = Xall[i];
  CUCHK(cudaMemsetAsync(ctx->d_flags.p, 0, 4 * sizeof(int), st));
  CUCHK(cudaMemsetAsync(ctx->d_Mmax.p, 0, sizeof(double), st));
  CUCHK(cudaMemsetAsync(ctx->d_blkacc.p, 0, 4 * CQG_NQC * sizeof(unsigned long long), st));
  const double cut32 = ctx->policy == CQG_PREC_MIXED ? ctx->fp32_cutoff : 0.0;
  ctx->launches = 0;
  {
    dim3 g((ctx->max_nsh + 127) / 128, ctx->max_nsh, ctx->nmol);
    k_blocknorm<<<g, 128, 0, st>>>(xl, ldx, mols, ctx->d_bf.p, ctx->d_sz.p, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, ctx->d_flags.p, 1e-12);
    CUCHK(cudaGetLastError());
    long long nn = ctx->Mtotal;
    int nb = (int)std::min<long long>((nn + 255) / 256, 1184);
    k_maxreduce<<<nb, 256, 0, st>>>(ctx->d_M.p, nn, ctx->d_Mmax.p);
    CUCHK(cudaGetLastError());
    ctx->launches += 2;
  }
  // 2. quartet lists
  Pairs P = make_pairs(ctx);
  {
    int nthr = 256, wpb = nthr / 32;
    int nb = (ctx->ntask + wpb - 1) / wpb;
    k_quartets<false><<<nb, nthr, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                            ctx->thresh,
                                            cut32, ctx->d_cnt.p, nullptr, nullptr, ctx->d_blkacc.p, 0, 0, 0, 0);
    CUCHK(cudaGetLastError());
    size_t scan_bytes = ctx->d_scan_tmp.n;
    CUCHK(cub::DeviceScan::ExclusiveSum(ctx->d_scan_tmp.p, scan_bytes, ctx->d_cnt.p, ctx->d_off.p, 2 * ctx->ntask, st));
    k_block_ranges<<<1, 128, 0, st>>>(ctx->bt, ctx->ntask, ctx->d_cnt.p, ctx->d_off.p, ctx->d_range.p, LLONG_MAX,
                                      ctx->d_flags.p);
    CUCHK(cudaGetLastError());
    ctx->launches += 2;
  }
  long long hr[4 * CQG_NQC];
  unsigned long long hacc[4 * CQG_NQC];
  int hflags[4];
  CUCHK(cudaMemcpyAsync(hr, ctx->d_range.p, sizeof(hr), cudaMemcpyDeviceToHost, st));
  CUCHK(cudaMemcpyAsync(hacc, ctx->d_blkacc.p, sizeof(hacc), cudaMemcpyDeviceToHost, st));
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
  long long total = hr[4 * CQG_NQC - 1];
  // The list is [FP64 part of every task][FP32 part of every task] ("virtual tasks"
  // 0 .. 2 ntask).  It is filled and consumed in chunks of at most `list_budget` quartets.
  const long long budget = std::max<long long>(ctx->list_budget, 1);
  std::vector<long long> chunk_vt;   // chunk boundaries in virtual tasks
  std::vector<long long> hoff, hcnt;
  const long long nvt = 2LL * ctx->ntask;
  if (total <= budget) {
    chunk_vt = {0, nvt};
  } else {
    hoff.resize(nvt);
    hcnt.resize(nvt);
    CUCHK(cudaMemcpyAsync(hoff.data(), ctx->d_off.p, nvt * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CUCHK(cudaMemcpyAsync(hcnt.data(), ctx->d_cnt.p, nvt * sizeof(long long), cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
    chunk_vt.push_back(0);
    long long start = 0;
    for (long long v = 0; v < nvt; ++v) {
      if (hoff[v] + hcnt[v] - start > budget && v > chunk_vt.back()) {
        chunk_vt.push_back(v);
        start = hoff[v];
      }
    }
    chunk_vt.push_back(nvt);
  }
  long long cap = std::min(total, budget);
  if (chunk_vt.size() > 2) {   // a single task may exceed the budget: size to the largest chunk
    cap = 0;
    for (size_t c = 0; c + 1 < chunk_vt.size(); ++c) {
      const long long v0 = chunk_vt[c], v1 = chunk_vt[c + 1];
      cap = std::max(cap, hoff[v1 - 1] + hcnt[v1 - 1] - hoff[v0]);
    }
  }
  if (ctx->d_qlist.reserve((size_t)std::max<long long>(cap, 1)) != cudaSuccess) {
    ctx->err = "quartet list allocation failed";
    return CQG_ERR_OOM;
  }
  ctx->stats.chunks = (long long)chunk_vt.size() - 1;
  if (ctx->d_G.reserve((size_t)ngroups * gsize) != cudaSuccess) return CQG_ERR_OOM;
  CUCHK(cudaMemsetAsync(ctx->d_G.p, 0, (size_t)ngroups * gsize * sizeof(double), st));
  DigestGroups dg;
  memset(&dg, 0, sizeof(dg));
  dg.ng = ngroups;
  dg.ldx = ldx;
  dg.batch = ctx->nmol > 1;
  dg.xoff = ctx->d_mxoff.p;
  dg.nbf = ctx->d_mnbf.p;
  for (int g = 0; g < ngroups; ++g) {
    dg.X[g] = Xg[g];
    dg.G[g] = ctx->d_G.p + (size_t)g * gsize;
    dg.sJ[g] = sJ[g];
    dg.sK[g] = sK[g];
  }
  memset(ctx->stats.class_quartets, 0, sizeof(ctx->stats.class_quartets));
  memset(ctx->stats.class_ms, 0, sizeof(ctx->stats.class_ms));
  double mflops = 0, mflops32 = 0;
  long long nprimq = 0, nq32 = 0;
  for (int k = 0; k < CQG_NQC; ++k) {
    const long long n64 = hr[2 * k + 1] - hr[2 * k];
    const long long n32 = hr[2 * (CQG_NQC + k) + 1] - hr[2 * (CQG_NQC + k)];
    ctx->stats.class_quartets[k] = n64 + n32;
    nq32 += n32;
    int i, j;
    qclass_split(k, i, j);
    const int la = kPairClass[i][0], lb = kPairClass[i][1], lc = kPairClass[j][0], ld = kPairClass[j][1];
    const double fp = md_v1_prim_flops(la, lb, lc, ld), fd = md_v1_digest_flops(la, lb, lc, ld);
    mflops += (double)hacc[4 * k] * fp + (double)n64 * fd;
    mflops32 += (double)hacc[4 * k + 2] * fp + (double)n32 * fd;
    nprimq += (long long)(hacc[4 * k + 1] + hacc[4 * k + 3]);
  }
  bool first_chunk = true;
  for (size_t ch = 0; ch + 1 < chunk_vt.size(); ++ch) {
    const long long vt0 = chunk_vt[ch], vt1 = chunk_vt[ch + 1];
    long long obase = 0;
    long long crange[4 * CQG_NQC];
    if (chunk_vt.size() > 2) {
      obase = hoff[vt0];
      for (int vb = 0; vb < 2 * CQG_NQC; ++vb) {
        const int prec = vb / CQG_NQC, b = vb % CQG_NQC;
        long long t0 = (long long)prec * ctx->ntask + ctx->bt.task_beg[b];
        long long t1 = (long long)prec * ctx->ntask + ctx->bt.task_beg[b + 1];
        t0 = std::max(t0, vt0);
        t1 = std::min(t1, vt1);
        if (t1 > t0) {
          crange[2 * vb] = hoff[t0] - obase;
          crange[2 * vb + 1] = hoff[t1 - 1] + hcnt[t1 - 1] - obase;
        } else {
          crange[2 * vb] = crange[2 * vb + 1] = 0;
        }
      }
      CUCHK(cudaMemcpyAsync(ctx->d_range.p, crange, sizeof(crange), cudaMemcpyHostToDevice, st));
    } else {
      for (int q = 0; q < 4 * CQG_NQC; ++q) crange[q] = hr[q];
    }
    {
      int nthr = 256, wpb = nthr / 32;
      int nb = (ctx->ntask + wpb - 1) / wpb;
      k_quartets<true><<<nb, nthr, 0, st>>>(ctx->bt, ctx->ntask, P, ctx->d_M.p, ctx->d_M.p + ctx->Mtotal, mols, ctx->d_shmol.p, ctx->d_Mmax.p,
                                             ctx->thresh,
                                             cut32, nullptr, ctx->d_off.p, ctx->d_qlist.p, nullptr, vt0, vt1, obase,
                                             (long long)ctx->d_qlist.n);
      CUCHK(cudaGetLastError());
      ctx->launches += 1;
    }
    if (ctx->timing && first_chunk) CUCHK(cudaEventRecord(ctx->ev[1], st));
    if (ctx->autotune_pending && chunk_vt.size() == 2) {
      cqg_status ts = autotune_shapes(ctx, crange, st, dg);
      if (ts != CQG_OK) return ts;
      ctx->autotune_pending = 0;
    }
    // 3. ERI + digest per class
    for (int k = 0; k < CQG_NQC; ++k) {
      const long long n64 = crange[2 * k + 1] - crange[2 * k];
      const long long n32 = crange[2 * (CQG_NQC + k) + 1] - crange[2 * (CQG_NQC + k)];
      if (n64 > 0) ctx->launches += 1;
      if (n32 > 0) ctx->launches += 1;
      if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[4 + 2 * k], st));
      cudaError_t e = kEriLaunch[k](ctx, k, n64, st, dg);
      if (e == cudaSuccess) e = kEriLaunch32[k](ctx, CQG_NQC + k, n32, st, dg);
      if (e != cudaSuccess) {
        ctx->err = std::string("eri kernel ") + cqg_class_name(k) + ": " + cudaGetErrorString(e);
        return CQG_ERR_CUDA;
      }
      if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[5 + 2 * k], st));
    }
    if (ctx->timing) {   // per-class device time, summed over chunks
      CUCHK(cudaStreamSynchronize(st));
      for (int k = 0; k < CQG_NQC; ++k) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev[4 + 2 * k], ctx->ev[5 + 2 * k]) == cudaSuccess)
          ctx->stats.class_ms[k] += ms;
      }
    }
    first_chunk = false;
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[2], st));
  // 4. AX += 0.5 (Gh + Gh^T)
  for (int g = 0; g < ngroups; ++g) {
    dim3 grid((ctx->max_nbf + 31) / 32, (ctx->max_nbf + 31) / 32, ctx->nmol), blk(32, 8);
    k_finalize<<<grid, blk, 0, st>>>(dg.G[g], mols, AXg[g], ldax);
    CUCHK(cudaGetLastError());
    ctx->launches += 1;
  }
  if (ctx->timing) CUCHK(cudaEventRecord(ctx->ev[3], st));
  ctx->stats.quartets = total;
  ctx->stats.quartets_fp32 = nq32;
  ctx->stats.model_flops = mflops + mflops32;
  ctx->stats.model_flops_fp32 = mflops32;
  ctx->stats.prim_quartets = nprimq;
  ctx->stats.launches = ctx->launches;
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
  if (on_device && ctx->graph_capacity > 0) return contract_graph(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ld, ld, st);
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
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  const int n = ctx->nbf;
  if (ld < n) {   // checked before PT is zeroed: nothing is written on a bad call
    ctx->err = "leading dimension below the number of basis functions";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
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

cqg_status cqg_one_e(cqg_ctx *ctx, int ncharge, const double *Z, const double *R, double *S, double *T, double *V,
                     int ld, int on_device, void *stream) {
  if (!ctx || ncharge < 0 || (ncharge > 0 && (!Z || !R)) || !S || !T || !V) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  const int n = ctx->nbf;
  if (ld < n) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (ctx->d_charges.reserve(4 * (size_t)std::max(ncharge, 1))) return CQG_ERR_OOM;
  std::vector<double> zr(4 * (size_t)std::max(ncharge, 1), 0.0);
  for (int c = 0; c < ncharge; ++c) {
    zr[c] = Z[c];
    zr[ncharge + 3 * c] = R[3 * c];
    zr[ncharge + 3 * c + 1] = R[3 * c + 1];
    zr[ncharge + 3 * c + 2] = R[3 * c + 2];
  }
  CUCHK(cudaMemcpyAsync(ctx->d_charges.p, zr.data(), zr.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  double *dS = S, *dT = T, *dV = V;
  int ldd = ld;
  if (!on_device) {
    if (ctx->d_oe.reserve(3 * (size_t)n * n)) return CQG_ERR_OOM;
    dS = ctx->d_oe.p;
    dT = dS + (size_t)n * n;
    dV = dT + (size_t)n * n;
    ldd = n;
  }
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  if (ctx->nmol != 1) {
    ctx->err = "cqg_one_e is for single-molecule contexts; use cqg_one_e_batch";
    return CQG_ERR_STATE;
  }
  const long long np = ctx->nallpairs;
  OneEMols om;
  memset(&om, 0, sizeof(om));
  k_one_e<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np, ncharge, ctx->d_charges.p,
                                                     (const double3 *)(ctx->d_charges.p + ncharge), ctx->d_boys.p, dS,
                                                     dT, dV, ldd, om);
  CUCHK(cudaGetLastError());
  if (!on_device) {
    double *outs[3] = {S, T, V};
    const double *ins[3] = {dS, dT, dV};
    for (int q = 0; q < 3; ++q)
      CUCHK(cudaMemcpy2DAsync(outs[q], ld * sizeof(double), ins[q], n * sizeof(double), n * sizeof(double), n,
                              cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
  }
  return CQG_OK;
}

cqg_status cqg_dipole(cqg_ctx *ctx, const double *origin, double *D, int ld, int on_device, void *stream) {
  if (!ctx || !origin || !D) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  if (ctx->nmol != 1) {
    ctx->err = "cqg_dipole is for single-molecule contexts";
    return CQG_ERR_STATE;
  }
  const int n = ctx->nbf;
  if (ld < n) {
    ctx->err = "leading dimension below the number of basis functions";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  double *dD = D;
  int ldd = ld;
  if (!on_device) {
    if (ctx->d_oe.reserve(3 * (size_t)n * n)) return CQG_ERR_OOM;
    dD = ctx->d_oe.p;
    ldd = n;
  }
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  const long long np = ctx->nallpairs;
  k_dipole<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np,
                                                      make_double3(origin[0], origin[1], origin[2]), dD, ldd, n);
  CUCHK(cudaGetLastError());
  if (!on_device) {
    for (int k = 0; k < 3; ++k)
      CUCHK(cudaMemcpy2DAsync(D + (size_t)k * ld * n, ld * sizeof(double), dD + (size_t)k * n * n,
                              n * sizeof(double), n * sizeof(double), n, cudaMemcpyDeviceToHost, st));
    CUCHK(cudaStreamSynchronize(st));
  }
  return CQG_OK;
}

cqg_status cqg_one_e_batch(cqg_ctx *ctx, const int *ncharge_per_mol, const double *Z, const double *R, double *S,
                           double *T, double *V, void *stream) {
  if (!ctx || !ncharge_per_mol || !Z || !R || !S || !T || !V) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const int nmol = ctx->nmol;
  std::vector<int> coff(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) coff[m + 1] = coff[m] + ncharge_per_mol[m];
  const int nc = coff[nmol];
  if (ctx->d_charges.reserve(4 * (size_t)std::max(nc, 1) + nmol + 1)) return CQG_ERR_OOM;
  std::vector<double> zr(4 * (size_t)std::max(nc, 1) + nmol + 1, 0.0);
  for (int c = 0; c < nc; ++c) {
    zr[c] = Z[c];
    zr[nc + 3 * c] = R[3 * c];
    zr[nc + 3 * c + 1] = R[3 * c + 1];
    zr[nc + 3 * c + 2] = R[3 * c + 2];
  }
  int *dcoff = (int *)(ctx->d_charges.p + 4 * (size_t)std::max(nc, 1));
  CUCHK(cudaMemcpyAsync(ctx->d_charges.p, zr.data(), 4 * (size_t)std::max(nc, 1) * sizeof(double),
                        cudaMemcpyHostToDevice, st));
  CUCHK(cudaMemcpyAsync(dcoff, coff.data(), (nmol + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  OneEMols om;
  om.shmol = ctx->d_shmol.p;
  om.xoff = ctx->d_mxoff.p;
  om.nbf = ctx->d_mnbf.p;
  om.coff = dcoff;
  om.batch = 1;
  const long long np = ctx->nallpairs;
  k_one_e<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np, nc, ctx->d_charges.p,
                                                     (const double3 *)(ctx->d_charges.p + nc), ctx->d_boys.p, S, T,
                                                     V, 0, om);
  CUCHK(cudaGetLastError());
  return CQG_OK;
}

cqg_status cqg_get_batch_layout(cqg_ctx *ctx, int *nbf_per_mol, long long *offset_per_mol, long long *packed) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  for (int m = 0; m < ctx->nmol; ++m) {
    if (nbf_per_mol) nbf_per_mol[m] = ctx->m_nbf[m];
    if (offset_per_mol) offset_per_mol[m] = ctx->m_xoff[m];
  }
  if (packed) *packed = ctx->packed;
  return CQG_OK;
}

cqg_status cqg_twoe_contract_direct_batch(cqg_ctx *ctx, int nmat, const double *const *X, double *const *AX,
                                          const int *types, const double *scale, const unsigned char *active,
                                          void *stream) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis_batch has not been called";
    return CQG_ERR_STATE;
  }
  if (nmat <= 0 || nmat > 8 || !X || !AX || !types || !scale) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned char all1 = 1;
  bool changed = false;
  for (int m = 0; m < ctx->nmol; ++m) {
    const unsigned char a = active ? (active[m] ? 1 : 0) : all1;
    if (a != ctx->h_active[m]) {
      ctx->h_active[m] = a;
      changed = true;
    }
  }
  if (changed && ctx->graph_capacity > 0) {
    ctx->err = "graph mode: change the active set with cqg_set_active outside the captured call";
    return CQG_ERR_STATE;
  }
  if (changed)
    CUCHK(cudaMemcpyAsync(ctx->d_active.p, ctx->h_active.data(), ctx->nmol, cudaMemcpyHostToDevice, st));
  const double *Xg[CQG_MAXG];
  double *AXg[CQG_MAXG];
  double sJ[CQG_MAXG], sK[CQG_MAXG];
  const double *Xu[8];
  int ng, nxu;
  cqg_status s = plan_groups(ctx, nmat, X, AX, types, scale, ng, Xg, AXg, sJ, sK, nxu, Xu);
  if (s != CQG_OK) return s;
  if (ctx->graph_capacity > 0) return contract_graph(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ctx->max_nbf, ctx->max_nbf, st);
  return contract_device(ctx, ng, Xg, AXg, sJ, sK, nxu, Xu, ctx->max_nbf, ctx->max_nbf, st);
}

cqg_status cqg_set_graph_mode(cqg_ctx *ctx, long long capacity, int max_groups) {
  if (!ctx || capacity < 0 || max_groups < 0 || max_groups > CQG_MAXG) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  ctx->graph_capacity = capacity;
  if (capacity > 0) {
    const size_t gsize = ctx->nmol > 1 ? (size_t)ctx->packed : (size_t)ctx->nbf * ctx->nbf;
    if (ctx->d_qlist.reserve((size_t)capacity) || ctx->d_G.reserve((size_t)std::max(max_groups, 1) * gsize)) {
      ctx->graph_capacity = 0;
      return CQG_ERR_OOM;
    }
  }
  return CQG_OK;
}

cqg_status cqg_graph_status(cqg_ctx *ctx, long long *quartets, int *overflow, int *nonfinite, int *asymmetric) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  CUCHK(cudaDeviceSynchronize());
  long long hr[4 * CQG_NQC];
  int fl[4];
  CUCHK(cudaMemcpy(fl, ctx->d_flags.p, sizeof(fl), cudaMemcpyDeviceToHost));
  CUCHK(cudaMemcpy(hr, ctx->d_range.p, sizeof(hr), cudaMemcpyDeviceToHost));
  if (quartets) *quartets = hr[4 * CQG_NQC - 1];
  if (overflow) *overflow = fl[2];
  if (nonfinite) *nonfinite = fl[0];
  if (asymmetric) *asymmetric = fl[1];
  return CQG_OK;
}

cqg_status cqg_set_active(cqg_ctx *ctx, const unsigned char *active) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  if (ctx->nshell == 0) return CQG_ERR_STATE;
  CUCHK(cudaSetDevice(ctx->device));
  for (int m = 0; m < ctx->nmol; ++m) ctx->h_active[m] = active ? (active[m] ? 1 : 0) : 1;
  CUCHK(cudaMemcpy(ctx->d_active.p, ctx->h_active.data(), ctx->nmol, cudaMemcpyHostToDevice));
  return CQG_OK;
}

cqg_status cqg_autotune_next(cqg_ctx *ctx) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  ctx->autotune_pending = 1;
  return CQG_OK;
}

cqg_status cqg_get_launch_shapes(cqg_ctx *ctx, int *cta_per_sm, int *warps_per_cta) {
  if (!ctx) return CQG_ERR_BAD_ARG;
  for (int k = 0; k < 2 * CQG_NQC; ++k) {
    if (cta_per_sm) cta_per_sm[k] = ctx->shape_cta[k];
    if (warps_per_cta) warps_per_cta[k] = ctx->shape_wpb[k];
  }
  return CQG_OK;
}

cqg_status cqg_get_stats(cqg_ctx *ctx, cqg_stats *out) {
  if (!ctx || !out) return CQG_ERR_BAD_ARG;
  CUCHK(cudaSetDevice(ctx->device));
  CUCHK(cudaDeviceSynchronize());
  cqg_stats &s = ctx->stats;
  if (ctx->timing) {
    float ms;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    s.ms_screen = ms;
    double eri = 0.0;
    for (int k = 0; k < CQG_NQC; ++k) eri += s.class_ms[k];
    s.ms_eri = eri;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[3]);
    s.ms_total = ms;

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

// ---- One-electron integrals that allocate nothing ---------------------------------------
// The point-charge table lives in a fixed module-scope device array instead of the
// context's growable buffer.  Its device address is resolved on the first such call of a
// context, with the context's device current, and kept in the context: a context never
// outlives its device's CUDA context (a cudaDeviceReset frees every buffer a context holds,
// so it is destroyed and created again), which keeps the address from going stale.
namespace {
// Z[0..n) followed by R[n..4n) (x, y, z per charge), as k_one_e reads it
__device__ __align__(256) double g_oe_charge_table[4 * CQG_ONE_E_NOALLOC_MAX_CHARGES];

// With ctx->device current: the device address of g_oe_charge_table on that device.
cqg_status oe_charge_table(cqg_ctx *ctx, double **out) {
  if (!ctx->oe_table) {
    void *p = nullptr;
    CUCHK(cudaGetSymbolAddress(&p, g_oe_charge_table));
    ctx->oe_table = (double *)p;
  }
  *out = ctx->oe_table;
  return CQG_OK;
}
}  // namespace

extern "C" {

cqg_status cqg_one_e_noalloc(cqg_ctx *ctx, int ncharge, const double *Z, const double *R, double *S, double *T,
                             double *V, int ld, void *stream) {
  if (!ctx || ncharge < 0 || (ncharge > 0 && (!Z || !R)) || !S || !T || !V) return CQG_ERR_BAD_ARG;
  if (ncharge > CQG_ONE_E_NOALLOC_MAX_CHARGES) {
    ctx->err = "cqg_one_e_noalloc: ncharge exceeds CQG_ONE_E_NOALLOC_MAX_CHARGES (4096)";
    return CQG_ERR_BAD_ARG;
  }
  if (ctx->nshell == 0) {
    ctx->err = "cqg_set_basis has not been called";
    return CQG_ERR_STATE;
  }
  if (ctx->nmol != 1) {
    ctx->err = "cqg_one_e_noalloc is for single-molecule contexts";
    return CQG_ERR_STATE;
  }
  if (ld < ctx->nbf) {
    ctx->err = "leading dimension below the number of basis functions";
    return CQG_ERR_BAD_ARG;
  }
  CUCHK(cudaSetDevice(ctx->device));
  double *tab = nullptr;
  const cqg_status s = oe_charge_table(ctx, &tab);
  if (s != CQG_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  // Z and R may be host or device pointers; the table is written in full for the
  // `ncharge` entries the kernel reads, so nothing in it has to start at zero.
  if (ncharge > 0) {
    CUCHK(cudaMemcpyAsync(tab, Z, (size_t)ncharge * sizeof(double), cudaMemcpyDefault, st));
    CUCHK(cudaMemcpyAsync(tab + ncharge, R, 3 * (size_t)ncharge * sizeof(double), cudaMemcpyDefault, st));
  }
  OneEShells sh;
  sh.L = ctx->d_shL.p;
  sh.nprim = ctx->d_shnp.p;
  sh.poff = ctx->d_shpoff.p;
  sh.bf = ctx->d_bf.p;
  sh.alpha = ctx->d_alpha.p;
  sh.coef = ctx->d_coef.p;
  sh.center = ctx->d_center.p;
  OneEMols om;
  memset(&om, 0, sizeof(om));
  const long long np = ctx->nallpairs;
  k_one_e<<<(unsigned)((np + 63) / 64), 64, 0, st>>>(sh, ctx->d_allpairs.p, np, ncharge, tab,
                                                     (const double3 *)(tab + ncharge), ctx->d_boys.p, S, T, V, ld,
                                                     om);
  CUCHK(cudaGetLastError());
  return CQG_OK;
}

}  // extern "C"
