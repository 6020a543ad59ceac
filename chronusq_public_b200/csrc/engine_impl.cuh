// Internals of the cqgpu engine shared by its translation units: device data layout,
// the screening / ERI / digest kernels (templates), the context structure and the
// class-kernel launchers.  engine.cu holds the C ABI; eri_part.cu instantiates the
// class kernels, a share of the quartet classes per translation unit, so that they
// compile in parallel.
#pragma once
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
#include "_gen/eri_gc_classes.cuh"
#include "eri_warp.cuh"

#define CQG_MAXL 3
#ifndef CQG_NPART
#define CQG_NPART 8          // translation units the class kernels are compiled in (eri_part.cu)
#endif
#define CQG_NPC ((CQG_MAXL + 1) * (CQG_MAXL + 2) / 2)       // pair classes
#define CQG_NQC (CQG_NPC * (CQG_NPC + 1) / 2)                // quartet classes
#define CQG_MAXG 4
#define CQG_NBUCKET 16   // ket buckets of a (molecule, pair class): the primitive-count bucket of the pair's group

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

// Members a sibling group of a pair class holds at most (larger families are split into
// groups of this size): s-s pairs 4 (two s shells of one contraction on each centre, or the
// three distinct pairs of one centre's two), p-s and d-s pairs 2, every other class 1 (not
// grouped: the classes whose sibling pairs keep one orientation, L_a > L_b, or are
// symmetric in a and b, s-s).
__host__ __device__ constexpr int sibling_cap(int la, int lb) {
  return (la == 0 && lb == 0) ? 4 : ((la == 1 || la == 2) && lb == 0) ? 2 : 1;
}

// Sibling-group quartet classes (generated sibling form EriClassGC<.., MB, MK>, MB and MK
// the member caps of the bra and ket pair classes).
template <int LA, int LB, int LC, int LD>
struct EriGroup {
  static constexpr bool ok = false;
  static constexpr int MB = 1, MK = 1;
};
#define CQG_GC_TRAIT(A, B, C, D, MB_, MK_)                                                            \
  template <>                                                                                       \
  struct EriGroup<A, B, C, D> {                                                                     \
    static constexpr bool ok = true;                                                                \
    static constexpr int MB = MB_, MK = MK_;                                                        \
    static_assert(MB_ == sibling_cap(A, B) && MK_ == sibling_cap(C, D), "member caps of the class"); \
  };
CQG_GC_EACH(CQG_GC_TRAIT)
#undef CQG_GC_TRAIT

__host__ __device__ constexpr int pair_class_c(int la, int lb) { return la * (la + 1) / 2 + lb; }
// quartet class index (bra pair class i >= ket pair class j, k = i(i+1)/2 + j)
__host__ __device__ constexpr int qclass_index(int la, int lb, int lc, int ld) {
  return pair_class_c(la, lb) * (pair_class_c(la, lb) + 1) / 2 + pair_class_c(lc, ld);
}

// quartet class k <-> (bra pair class i, ket pair class j), i >= j, k = i(i+1)/2 + j
static inline void qclass_split(int k, int &i, int &j) {
  i = 0;
  while ((i + 1) * (i + 2) / 2 <= k) ++i;
  j = k - i * (i + 1) / 2;
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
  const int *molgbk;             // the same in group index space: first group of each bucket
};
struct Pairs {
  const int2 *sh;       // (shell a, shell b), internal orientation L_a >= L_b
  const double *Q;      // Schwarz bound
  const int *poff;      // first primitive pair
  const int *np;        // number of primitive pairs (after primitive screening)
  const int *kk;        // nprim(a) * nprim(b) of the contracted shells (model count)
  const PrimPair *prim;
  // Sibling groups: pairs whose shells have the same centres, angular momenta and
  // exponents (segmented copies of one general contraction) and differ only in their
  // contraction coefficients.  The members of a group are consecutive pairs, led by the
  // first.  Group g (group index space, in pair order) is led by pair glead[g]; gQ[g] is
  // the largest Q of its members and Qc[i] that of pair i's group (non-increasing within a
  // primitive bucket, so it serves the coarse range searches).
  const double *Qc;
  const int *glead;
  const double *gQ;
  // Per pair (meaningful for leaders): gsz members (0 for the other members), and the
  // group's unit-coefficient primitive pairs gprim[gpoff .. gpoff + gnp) (the union of the
  // members' screened primitive pairs) with the members' coefficient products
  // gw[gwoff + m * gnp + i], m < the member cap of the pair class (zero rows past gsz).
  const int *gsz;
  const int *gpoff;
  const int *gnp;
  const int *gwoff;
  const PrimPair *gprim;
  const double *gw;
  // Member masks of the sibling-group list entries (bit 4 i + j: bra member i with ket
  // member j), parallel to the quartet list.
  const unsigned short *qmask;
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
static __global__ void k_blocknorm(XList xl, int ldx, Mols mols, const int *__restrict__ bf,
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

static __global__ void k_maxreduce(const double *__restrict__ M, long long n, double *__restrict__ out) {
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
  int grouped[CQG_NQC];        // tasks are bra sibling groups
  int gbra_beg[CQG_NQC];       // first bra group (group index) of a grouped block
  int min_members[CQG_NQC];    // grouped: member quartets a sibling entry holds at least
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
// m12 = M(s1, s2) is the bra's own, the same for every ket, and mcd = M(s3, s4) the ket's
// own, read from the per-pair copy Mpair (consecutive kets: a coalesced load).
__device__ __forceinline__ double quartet_bound(const double *__restrict__ col1, const double *__restrict__ col2,
                                                double m12, double mcd, int shoff, int2 cd, double qab, double qcd) {
  const int s3 = cd.x - shoff, s4 = cd.y - shoff;
  double m = fmax(m12, col1[s4]);
  m = fmax(m, col2[s4]);
  m = fmax(m, mcd);
  m = fmax(m, col1[s3]);
  m = fmax(m, col2[s3]);
  return m * qab * qcd;
}

// Mpair[i] = M(a, b) of shell pair i (its own block norm; molecule-local indices).
static __global__ void k_pairnorm(const int2 *__restrict__ sh, int npairs, Mols mols, const int *__restrict__ shmol,
                                  const double *__restrict__ M, double *__restrict__ Mpair) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npairs) return;
  const int2 ab = sh[i];
  const int mol = shmol[ab.x];
  const int nsh = mols.nsh[mol], shoff = mols.shoff[mol];
  Mpair[i] = M[mols.Moff[mol] + (ab.x - shoff) + (size_t)(ab.y - shoff) * nsh];
}

// Per-block screening tallies in blkacc[kBlkAcc * blk + ...]: model primitive quartets
// (sum of Ka Kb Kc Kd) and executed primitive quartets of the FP64 and FP32 lists, then the
// number of contracted quartets of each (a sibling-group entry holds several).
constexpr int kBlkAcc = 6;

// The quartet list is laid out by virtual task v = part * ntask + task, part 0 / 1 = the
// FP64 / FP32 pair entries (one quartet each), part 2 / 3 = the FP64 / FP32 sibling-group
// entries; work list vb = part * CQG_NQC + class is the range of one part of one class.
constexpr int kListParts = 4;
#define CQG_NLIST (kListParts * CQG_NQC)
constexpr int kRangeThreads = 256;   // k_block_ranges: one thread per work list
static_assert(CQG_NLIST <= kRangeThreads, "k_block_ranges needs a thread per work list");

// exclusive prefix sum over the warp's lanes and the warp's total
__device__ __forceinline__ unsigned warp_excl_scan(unsigned x, unsigned &total) {
  const int lane = threadIdx.x & 31;
  unsigned v = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  total = __shfl_sync(0xffffffffu, v, 31);
  return v - x;
}

// Count (FILL=false) or write (FILL=true) the passing quartets of each task.  One warp
// per task; ket pairs scanned in ascending order, survivors compacted in lane order so the
// list is deterministic.  Quartets whose bound is below `cut32` go to the FP32 parts; the
// rest to the FP64 parts.  Counts cnt[v], offsets off[v] per virtual task v.
//
// In a grouped block a task is one bra sibling group and each lane takes one ket group:
// every member quartet (bra member i, ket member j) gets the exact test above.  A pair of
// groups with at least bt.min_members[blk] member quartets becomes one sibling entry (bra
// leader, ket leader) per precision, with the mask of its members that passed at that
// precision; the members of a smaller pair of groups become pair entries of their own.  So
// the contracted quartets, their count and their precision are those of the pair-level
// lists.  In a diagonal block (bra class = ket class) ket group <= bra group, and within one
// group ket member <= bra member, so every unordered pair of pairs is taken once.
//
// Tasks take the class's bra pairs (groups) from the last: the pairs are ordered by
// primitive-count bucket, so each class list starts with its heaviest quartets and the
// work queues hand out the light ones at the end of a launch.
struct ScreenTally {
  unsigned long long km64 = 0, ke64 = 0, km32 = 0, ke32 = 0, nq64 = 0, nq32 = 0;
};

// Survivor-mask cache between the two screening passes: the count pass stores, per task and
// per 32-ket step, the FP64 and FP32 survivor ballots (one uint2) at the task's slot in
// `masks`; the fill pass reads them instead of testing the bounds again.  A task whose
// steps do not fit in the buffer gets slot -1 and the fill pass tests its bounds itself.
static_assert(CQG_NBUCKET <= 32, "screen_pair_task searches one bucket per lane");
constexpr long long kMaskStepsInitial = 1ll << 22;   // 32 MiB; grown to what a call used
constexpr long long kMaskStepsMax = 1ll << 28;       // 2 GiB
struct MaskCache {
  uint2 *masks;
  unsigned long long *head;   // next free step (zeroed before the count pass)
  long long *slot;            // per task: first step, or -1
  long long cap;              // steps the buffer holds
};

template <bool FILL>
__device__ __forceinline__ void screen_pair_task(const BlockTable &bt, int blk, int t, int task, const Pairs &P,
                                                 const double *__restrict__ M, const double *__restrict__ MT,
                                                 const double *__restrict__ Mpair, const Mols &mols,
                                                 const int *__restrict__ shmol, double mm, double thresh,
                                                 double cut32, const bool (&dop)[kListParts],
                                                 const long long (&base)[kListParts], long long (&cpart)[kListParts],
                                                 uint2 *__restrict__ qlist, long long cap, const MaskCache &mc,
                                                 ScreenTally &ty) {
  const int lane = threadIdx.x & 31;
  const int bra = bt.bra_beg[blk] + t;
  const double qb = P.Q[bra];
  if (!(qb * mm > 0.0)) {
    if (!FILL && lane == 0) mc.slot[task] = -1;
    return;
  }
  const double cut = thresh / (qb * mm) * (1.0 - 1e-12);
  const int2 ab = P.sh[bra];
  const int mol = shmol[ab.x];
  if (!mols.active[mol]) {
    if (!FILL && lane == 0) mc.slot[task] = -1;
    return;
  }
  const int nsh = mols.nsh[mol], shoff = mols.shoff[mol];
  const double *Mm = M + mols.Moff[mol];
  const double *col1 = MT + mols.Moff[mol] + (size_t)(ab.x - shoff) * nsh;
  const double *col2 = MT + mols.Moff[mol] + (size_t)(ab.y - shoff) * nsh;
  const double m12 = Mm[(ab.x - shoff) + (size_t)(ab.y - shoff) * nsh];
  const int *bkt = mols.molbk + ((size_t)mol * CQG_NPC + bt.ket_class[blk]) * (CQG_NBUCKET + 1);
  const unsigned long long kkb = (unsigned long long)P.kk[bra], npb = (unsigned long long)P.np[bra];
  const unsigned below = (1u << lane) - 1u;
  // coarse range of every bucket at once: lane b < CQG_NBUCKET searches bucket b
  int my_kb = 0, my_kend = 0;
  if (lane < CQG_NBUCKET) {
    const int kb = bkt[lane], ke = bkt[lane + 1];
    int kend = kb;
    if (ke > kb) {
      kend = kb + coarse_range(P.Qc, kb, ke - kb, cut);
      if (bt.diag[blk]) kend = min(kend, bra + 1);   // unique pairs of pairs: ket <= bra
    }
    my_kb = kb;
    my_kend = max(kend, kb);
  }
  // the task's slot in the mask cache: the count pass reserves one step per 32 kets
  long long slot = -1;
  if (!FILL) {
    unsigned steps;
    warp_excl_scan((unsigned)((my_kend - my_kb + 31) >> 5), steps);
    if (lane == 0) {
      if (steps > 0) {
        const unsigned long long s0 = atomicAdd(mc.head, (unsigned long long)steps);
        slot = (long long)(s0 + steps) <= mc.cap ? (long long)s0 : -1;
      }
      mc.slot[task] = slot;
    }
    slot = __shfl_sync(0xffffffffu, slot, 0);
  } else {
    slot = mc.slot[task];
  }
  long long step = 0;
  for (int bk = 0; bk < CQG_NBUCKET; ++bk) {
    const int kb = __shfl_sync(0xffffffffu, my_kb, bk), kend = __shfl_sync(0xffffffffu, my_kend, bk);
    for (int k0 = kb; k0 < kend; k0 += 32, ++step) {
      const int ket = k0 + lane;
      unsigned b64, b32;
      if (FILL && slot >= 0) {   // survivors from the count pass
        const uint2 m = mc.masks[slot + step];
        b64 = m.x;
        b32 = m.y;
      } else {
        bool hi = false, lo = false;
        if (ket < kend) {
          const double bnd = quartet_bound(col1, col2, m12, Mpair[ket], shoff, P.sh[ket], qb, P.Q[ket]);
          const bool pass = bnd >= thresh;
          lo = pass && bnd < cut32;
          hi = pass && !lo;
        }
        b64 = __ballot_sync(0xffffffffu, hi);
        b32 = __ballot_sync(0xffffffffu, lo);
        if (!FILL && slot >= 0 && lane == 0) mc.masks[slot + step] = make_uint2(b64, b32);
      }
      const bool hi = (b64 >> lane) & 1u, lo = (b32 >> lane) & 1u;
      if (FILL) {
        if (hi && dop[0]) {
          const long long pos = base[0] + cpart[0] + __popc(b64 & below);
          if (pos < cap) qlist[pos] = make_uint2((unsigned)bra, (unsigned)ket);
        }
        if (lo && dop[1]) {
          const long long pos = base[1] + cpart[1] + __popc(b32 & below);
          if (pos < cap) qlist[pos] = make_uint2((unsigned)bra, (unsigned)ket);
        }
      } else {
        if (hi) {
          ty.km64 += (unsigned long long)P.kk[ket];
          ty.ke64 += (unsigned long long)P.np[ket];
        }
        if (lo) {
          ty.km32 += (unsigned long long)P.kk[ket];
          ty.ke32 += (unsigned long long)P.np[ket];
        }
      }
      cpart[0] += __popc(b64);
      cpart[1] += __popc(b32);
    }
  }
  if (!FILL) {   // the bra's factors are common to the task's quartets
    ty.km64 *= kkb;
    ty.ke64 *= npb;
    ty.km32 *= kkb;
    ty.ke32 *= npb;
    ty.nq64 = (unsigned long long)cpart[0];
    ty.nq32 = (unsigned long long)cpart[1];
  }
}

template <bool FILL>
__device__ __forceinline__ void screen_group_task(const BlockTable &bt, int blk, int t, const Pairs &P,
                                                  const double *__restrict__ MT, const double *__restrict__ Mpair,
                                                  const Mols &mols, const int *__restrict__ shmol, double mm,
                                                  double thresh, double cut32, const bool (&dop)[kListParts],
                                                  const long long (&base)[kListParts],
                                                  long long (&cpart)[kListParts], uint2 *__restrict__ qlist,
                                                  unsigned short *__restrict__ qmask, long long cap,
                                                  ScreenTally &ty) {
  const int lane = threadIdx.x & 31;
  const int gbra = bt.gbra_beg[blk] + t;
  const int bra = P.glead[gbra];
  const int mb = P.gsz[bra];
  const int min_members = bt.min_members[blk];
  const double qb = P.gQ[gbra];
  if (!(qb * mm > 0.0)) return;
  const double cut = thresh / (qb * mm) * (1.0 - 1e-12);
  const double tcut = thresh * (1.0 - 1e-12);   // margin for the rounding of the Q products
  const int mol = shmol[P.sh[bra].x];
  if (!mols.active[mol]) return;
  const int nsh = mols.nsh[mol], shoff = mols.shoff[mol];
  const double *MTm = MT + mols.Moff[mol];
  const int *bkt = mols.molgbk + ((size_t)mol * CQG_NPC + bt.ket_class[blk]) * (CQG_NBUCKET + 1);
  const unsigned below = (1u << lane) - 1u;
  for (int bk = 0; bk < CQG_NBUCKET; ++bk) {
    const int kb = bkt[bk], ke = bkt[bk + 1];
    if (ke <= kb) continue;
    int kend = kb + coarse_range(P.gQ, kb, ke - kb, cut);
    if (bt.diag[blk]) kend = min(kend, gbra + 1);   // ket group <= bra group
    for (int k0 = kb; k0 < kend; k0 += 32) {
      const int kx = k0 + lane;   // ket group
      int ket = 0;
      unsigned m64 = 0, m32 = 0;  // member masks, bit 4 i + j
      bool sib = false;
      if (kx < kend) {
        ket = P.glead[kx];
        const int mk = P.gsz[ket];
        const bool same = bt.diag[blk] && kx == gbra;
        sib = mb * mk > 1 && (same ? mb * (mb + 1) / 2 : mb * mk) >= min_members;
        const double qk = P.gQ[kx];
        for (int i = 0; i < mb; ++i) {
          const int bi = bra + i;
          const double qi = P.Q[bi];
          // the bound of each member quartet is at most Mmax Q_i Q_j: skip the six norms where
          // that already falls short (the groups' coarse range holds their largest Q)
          if (qi * qk * mm < tcut) continue;
          const int2 abi = P.sh[bi];
          const double *c1 = MTm + (size_t)(abi.x - shoff) * nsh;
          const double *c2 = MTm + (size_t)(abi.y - shoff) * nsh;
          const double mi = Mpair[bi];
          const int jmax = same ? min(mk, i + 1) : mk;
          for (int j = 0; j < jmax; ++j) {
            const int kj = ket + j;
            const double qj = P.Q[kj];
            if (qi * qj * mm < tcut) continue;
            const double bnd = quartet_bound(c1, c2, mi, Mpair[kj], shoff, P.sh[kj], qi, qj);
            if (bnd < thresh) continue;
            const unsigned bit = 1u << (4 * i + j);
            if (bnd < cut32) m32 |= bit; else m64 |= bit;
            if (!FILL) {
              const unsigned long long kq = (unsigned long long)P.kk[bi] * (unsigned long long)P.kk[kj];
              // executed primitive quartets of a member quartet evaluated on its own
              const unsigned long long eq =
                  sib ? 0ull : (unsigned long long)P.np[bi] * (unsigned long long)P.np[kj];
              if (bnd < cut32) {
                ty.km32 += kq;
                ty.ke32 += eq;
              } else {
                ty.km64 += kq;
                ty.ke64 += eq;
              }
            }
          }
        }
        if (!FILL) {
          if (sib) {   // a sibling entry evaluates the groups' shared primitive pairs once
            const unsigned long long gq = (unsigned long long)P.gnp[bra] * (unsigned long long)P.gnp[ket];
            if (m64) ty.ke64 += gq;
            if (m32) ty.ke32 += gq;
          }
          ty.nq64 += (unsigned long long)__popc(m64);
          ty.nq32 += (unsigned long long)__popc(m32);
        }
      }
      // pair entries (one per member quartet) of parts 0 and 1: several per lane
      const unsigned n0 = sib ? 0u : (unsigned)__popc(m64), n1 = sib ? 0u : (unsigned)__popc(m32);
      unsigned t0, t1;
      const unsigned e0 = warp_excl_scan(n0, t0), e1 = warp_excl_scan(n1, t1);
      // sibling entries of parts 2 and 3: at most one per lane
      const unsigned b2 = __ballot_sync(0xffffffffu, sib && m64), b3 = __ballot_sync(0xffffffffu, sib && m32);
      if (FILL) {
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          unsigned m = p == 0 ? (sib ? 0u : m64) : (sib ? 0u : m32);
          if (!m || !dop[p]) continue;
          long long pos = base[p] + cpart[p] + (p == 0 ? e0 : e1);
          while (m) {   // member quartets in bit order
            const int bit = __ffs(m) - 1;
            m &= m - 1;
            if (pos < cap) qlist[pos] = make_uint2((unsigned)(bra + (bit >> 2)), (unsigned)(ket + (bit & 3)));
            ++pos;
          }
        }
        if (sib && m64 && dop[2]) {
          const long long pos = base[2] + cpart[2] + __popc(b2 & below);
          if (pos < cap) {
            qlist[pos] = make_uint2((unsigned)bra, (unsigned)ket);
            qmask[pos] = (unsigned short)m64;
          }
        }
        if (sib && m32 && dop[3]) {
          const long long pos = base[3] + cpart[3] + __popc(b3 & below);
          if (pos < cap) {
            qlist[pos] = make_uint2((unsigned)bra, (unsigned)ket);
            qmask[pos] = (unsigned short)m32;
          }
        }
      }
      cpart[0] += t0;
      cpart[1] += t1;
      cpart[2] += __popc(b2);
      cpart[3] += __popc(b3);
    }
  }
}

// Four CTAs of 256 threads per SM (64 registers; a few bytes of spills): the latency-bound
// screening runs 3.54 -> 3.02 ms per (H2O)_32 build against three CTAs at 80 registers.
template <bool FILL>
__global__ void __launch_bounds__(256, 4) k_quartets(BlockTable bt, int ntask, Pairs P, const double *__restrict__ M,
                                                  const double *__restrict__ MT, const double *__restrict__ Mpair,
                                                  Mols mols, const int *__restrict__ shmol,
                                                  const double *__restrict__ Mmax, double thresh,
                                                  double cut32, long long *__restrict__ cnt,
                                                  const long long *__restrict__ off, uint2 *__restrict__ qlist,
                                                  unsigned short *__restrict__ qmask,
                                                  unsigned long long *__restrict__ blkacc, long long vt0,
                                                  long long vt1, long long obase, long long cap, MaskCache mc) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ntask) return;
  // fill pass: only the parts (virtual tasks part * ntask + warp) inside the chunk
  bool dop[kListParts];
  bool any = false;
#pragma unroll
  for (int p = 0; p < kListParts; ++p) {
    const long long v = (long long)p * ntask + warp;
    dop[p] = !FILL || (v >= vt0 && v < vt1);
    any = any || dop[p];
  }
  if (FILL && !any) return;
  const int blk = find_block(bt, warp);
  const int t = bt.task_beg[blk + 1] - 1 - warp;   // heaviest bra first
  long long base[kListParts], cpart[kListParts];
#pragma unroll
  for (int p = 0; p < kListParts; ++p) {
    base[p] = FILL ? off[(long long)p * ntask + warp] - obase : 0;
    cpart[p] = 0;
  }
  ScreenTally ty;
  const double mm = *Mmax;
  if (bt.grouped[blk])
    screen_group_task<FILL>(bt, blk, t, P, MT, Mpair, mols, shmol, mm, thresh, cut32, dop, base, cpart, qlist,
                            qmask, cap, ty);
  else
    screen_pair_task<FILL>(bt, blk, t, warp, P, M, MT, Mpair, mols, shmol, mm, thresh, cut32, dop, base, cpart,
                           qlist, cap, mc, ty);
  if (!FILL) {
    for (int o = 16; o > 0; o >>= 1) {
      ty.km64 += __shfl_xor_sync(0xffffffffu, ty.km64, o);
      ty.ke64 += __shfl_xor_sync(0xffffffffu, ty.ke64, o);
      ty.km32 += __shfl_xor_sync(0xffffffffu, ty.km32, o);
      ty.ke32 += __shfl_xor_sync(0xffffffffu, ty.ke32, o);
    }
    if (bt.grouped[blk]) {   // pair tasks count whole warps already
      for (int o = 16; o > 0; o >>= 1) {
        ty.nq64 += __shfl_xor_sync(0xffffffffu, ty.nq64, o);
        ty.nq32 += __shfl_xor_sync(0xffffffffu, ty.nq32, o);
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int p = 0; p < kListParts; ++p) cnt[(long long)p * ntask + warp] = cpart[p];
      unsigned long long *acc = blkacc + kBlkAcc * blk;
      if (ty.nq64) {
        atomicAdd(acc + 0, ty.km64);
        atomicAdd(acc + 1, ty.ke64);
        atomicAdd(acc + 4, ty.nq64);
      }
      if (ty.nq32) {
        atomicAdd(acc + 2, ty.km32);
        atomicAdd(acc + 3, ty.ke32);
        atomicAdd(acc + 5, ty.nq32);
      }
    }
  }
}

// Ranges [beg, end) of the quartet list per work list vb = part * nblk + block from the
// per-task counts and offsets (virtual task part * ntask + task).
static __global__ void k_block_ranges(BlockTable bt, int ntask, const long long *__restrict__ cnt,
                               const long long *__restrict__ off, long long *__restrict__ range, long long cap,
                               int *__restrict__ flags) {
  int vb = threadIdx.x;
  const long long nv = (long long)kListParts * ntask;
  if (vb == 0 && ntask > 0 && off[nv - 1] + cnt[nv - 1] > cap) flags[2] = 1;   // list overflow
  if (vb >= kListParts * bt.nblk) return;
  const int part = vb / bt.nblk, b = vb % bt.nblk;
  const long long t0 = (long long)part * ntask + bt.task_beg[b], t1 = (long long)part * ntask + bt.task_beg[b + 1];
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

// Work queue: the class's quartet range [beg, end) is consumed in chunks of `chunk`
// quartets (a multiple of 32), each claimed by one warp with an atomic add on the list's
// head counter qhead[blk] (zeroed before the launch), so warps that drew cheap quartets
// take more chunks instead of idling at the tail of a static split.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_jk_list(const uint2 *__restrict__ ql, const long long *__restrict__ range, int blk,
                                            const Pairs &P, const Shells &S, const double *__restrict__ boys_g,
                                            const DigestGroups &dg, unsigned long long *__restrict__ qhead,
                                            int chunk) {
  __shared__ __align__(16) double boys[BOYS_NT * BOYS_SROW];
  stage_boys<LA + LB + LC + LD>(boys_g, boys);
  __syncthreads();
  const long long beg = range[2 * blk], end = range[2 * blk + 1];
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(qhead + blk, (unsigned long long)chunk);
    c0 = __shfl_sync(0xffffffffu, c0, 0);
    const long long cfirst = beg + (long long)c0;
    if (cfirst >= end) return;   // the whole list is claimed
    const long long cend = min(cfirst + (long long)chunk, end);
    for (long long wfirst = cfirst; wfirst < cend; wfirst += 32)
      eri_jk_one<LA, LB, LC, LD, T>(ql, wfirst + lane, wfirst, cend, P, S, boys, dg);
  }
}

template <int LA, int LB, int LC, int LD, typename T>
__global__ void __launch_bounds__(kEriThreads) k_eri_jk(const uint2 *__restrict__ ql, const long long *__restrict__ range,
                                                int blk, Pairs P, Shells S, const double *__restrict__ boys_g,
                                                DigestGroups dg, unsigned long long *__restrict__ qhead, int chunk) {
  eri_jk_list<LA, LB, LC, LD, T>(ql, range, blk, P, S, boys_g, dg, qhead, chunk);
}

// Classes whose kernel is compiled for MB resident CTAs per SM (launch bounds with a
// minimum block count; the other classes keep the compiler's own register choice).
// Measured on (H2O)_32 cc-pVDZ against the kernels without the minimum: (ps|ps) 151 -> 128
// registers 4.3 % faster, (pp|ss) 157 -> 128 2.9 %, (ds|ps) 199 -> 168 2.8 %; (ps|ss) at
// five CTAs (95 registers) no faster, (ss|ss) at five (96, spilling) 17 % slower.
template <int LA, int LB, int LC, int LD>
struct EriMinBlocks {
  static constexpr int v = 0;
};
template <>
struct EriMinBlocks<1, 0, 1, 0> {
  static constexpr int v = 4;
};
template <>
struct EriMinBlocks<1, 1, 0, 0> {
  static constexpr int v = 4;
};
template <>
struct EriMinBlocks<2, 0, 1, 0> {
  static constexpr int v = 3;
};

template <int LA, int LB, int LC, int LD, typename T, int MB>
__global__ void __launch_bounds__(kEriThreads, MB) k_eri_jk_mb(const uint2 *__restrict__ ql,
                                                       const long long *__restrict__ range, int blk, Pairs P,
                                                       Shells S, const double *__restrict__ boys_g, DigestGroups dg,
                                                       unsigned long long *__restrict__ qhead, int chunk) {
  eri_jk_list<LA, LB, LC, LD, T>(ql, range, blk, P, S, boys_g, dg, qhead, chunk);
}

// One list entry (pair quartet) per lane with the class's per-thread code and its digest.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_jk_plain(const uint2 e, const bool valid, const Pairs &P, const Shells &S,
                                             const double *boys, const DigestGroups &dg) {
  constexpr int NA = nfun_c(LA), NB = nfun_c(LB), NC = nfun_c(LC), ND = nfun_c(LD);
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

// One sibling-group entry per lane: the generated sibling form evaluates the MB x MK member
// quartets (bra members leader e.x + i, ket members e.y + j) from one pass over the groups'
// primitive pairs, then each member quartet of the entry's mask is digested as a quartet of
// its own.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_jk_group(const uint2 e, const bool valid, const unsigned mask, const Pairs &P,
                                             const Shells &S, const double *boys, const DigestGroups &dg) {
  constexpr int NA = nfun_c(LA), NB = nfun_c(LB), NC = nfun_c(LC), ND = nfun_c(LD);
  constexpr int NQ = NA * NB * NC * ND;
  constexpr int MB = EriGroup<LA, LB, LC, LD>::MB, MK = EriGroup<LA, LB, LC, LD>::MK;
  const int mb = P.gsz[e.x], mk = P.gsz[e.y];
  double v[MB * MK * NQ];
  if (valid) {
    const int2 ab = P.sh[e.x], cd = P.sh[e.y];
    const double3 A = S.center[ab.x], B = S.center[ab.y], C = S.center[cd.x], D = S.center[cd.y];
    const PrimPair *bp = P.gprim + P.gpoff[e.x], *kp = P.gprim + P.gpoff[e.y];
    const double *bw = P.gw + P.gwoff[e.x], *kw = P.gw + P.gwoff[e.y];
    if constexpr (sizeof(T) == sizeof(double)) {
      EriClassGC<LA, LB, LC, LD, MB, MK>::template run<double>(bp, bw, P.gnp[e.x], kp, kw, P.gnp[e.y], A, B, C, D,
                                                               boys, v);
    } else {
      T vt[MB * MK * NQ];
      EriClassGC<LA, LB, LC, LD, MB, MK>::template run<T>(bp, bw, P.gnp[e.x], kp, kw, P.gnp[e.y], A, B, C, D, boys,
                                                          vt);
#pragma unroll
      for (int k = 0; k < MB * MK * NQ; ++k) v[k] = (double)vt[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < MB * MK * NQ; ++k) v[k] = 0.0;
  }
  const unsigned bra0 = __shfl_sync(0xffffffffu, e.x, 0);
  const bool uniform = __all_sync(0xffffffffu, e.x == bra0);
#pragma unroll
  for (int i = 0; i < MB; ++i) {
#pragma unroll
    for (int j = 0; j < MK; ++j) {
      const bool mv = valid && ((mask >> (4 * i + j)) & 1u);
      if (!__any_sync(0xffffffffu, mv)) continue;
      // members past the group's size are never in the mask; their lanes address the leader
      const int pa = i < mb ? (int)e.x + i : (int)e.x;
      const int pc = j < mk ? (int)e.y + j : (int)e.y;
      const int2 ab = P.sh[pa], cd = P.sh[pc];
      const double deg = (ab.x == ab.y ? 1.0 : 2.0) * (cd.x == cd.y ? 1.0 : 2.0) * (pa == pc ? 1.0 : 2.0);
      digest<NA, NB, NC, ND>(v + (i * MK + j) * NQ, deg, S.bf[ab.x], S.bf[ab.y], S.bf[cd.x], S.bf[cd.y], dg, mv,
                             uniform, S.mol[ab.x]);
    }
  }
}

template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_jk_one(const uint2 *__restrict__ ql, long long i, long long wfirst, long long end,
                                           const Pairs &P, const Shells &S, const double *boys,
                                           const DigestGroups &dg) {
  const bool valid = i < end;
  const uint2 e = ql[valid ? i : wfirst];
  eri_jk_plain<LA, LB, LC, LD, T>(e, valid, P, S, boys, dg);
}

// Sibling-group list of class (LA LB|LC LD): the work queue and persistent grid of
// k_eri_jk, one entry (bra group, ket group, member mask) per thread, NT threads per CTA
// (64 lets one more CTA of these register-heavy kernels reside on an SM).
template <int LA, int LB, int LC, int LD, typename T, int NT>
__global__ void __launch_bounds__(NT) k_eri_gc(const uint2 *__restrict__ ql, const long long *__restrict__ range,
                                                int blk, Pairs P, Shells S, const double *__restrict__ boys_g,
                                                DigestGroups dg, unsigned long long *__restrict__ qhead, int chunk) {
  __shared__ __align__(16) double boys[BOYS_NT * BOYS_SROW];
  stage_boys<LA + LB + LC + LD>(boys_g, boys);
  __syncthreads();
  const long long beg = range[2 * blk], end = range[2 * blk + 1];
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long c0 = 0;
    if (lane == 0) c0 = atomicAdd(qhead + blk, (unsigned long long)chunk);
    c0 = __shfl_sync(0xffffffffu, c0, 0);
    const long long cfirst = beg + (long long)c0;
    if (cfirst >= end) return;   // the whole list is claimed
    const long long cend = min(cfirst + (long long)chunk, end);
    for (long long wfirst = cfirst; wfirst < cend; wfirst += 32) {
      const long long i = wfirst + lane;
      const bool valid = i < cend;
      const uint2 e = ql[valid ? i : wfirst];
      const unsigned mask = valid ? (unsigned)P.qmask[i] : 0u;
      eri_jk_group<LA, LB, LC, LD, T>(e, valid, mask, P, S, boys, dg);
    }
  }
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
                                                     double *__restrict__ Qout, unsigned long long *__restrict__ qhead,
                                                     int qpw) {
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
  // list mode: each warp claims `qpw` quartets at a time from the work queue (head counter
  // qhead[blk]); Schwarz mode: a static split of the pairs over the warps
  const long long stride = (long long)gridDim.x * (blockDim.x >> 5);
  long long q = SCHWARZ ? beg + (long long)blockIdx.x * (blockDim.x >> 5) + wid : end;
  long long qend = end;
  for (;;) {
    if (SCHWARZ) {
      if (q >= end) break;
    } else if (q >= qend) {
      unsigned long long c0 = 0;
      if (lane == 0) c0 = atomicAdd(qhead + blk, (unsigned long long)qpw);
      c0 = __shfl_sync(0xffffffffu, c0, 0);
      q = beg + (long long)c0;
      if (q >= end) break;
      qend = min(q + (long long)qpw, end);
    }
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
      q += stride;
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
    ++q;
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
static __global__ void k_finalize(const double *__restrict__ Gh0, Mols mols, double *__restrict__ AX0, int ldax) {
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
  int shape_cta[CQG_NLIST] = {0};
  int shape_wpb[CQG_NLIST] = {0};
  // quartets a warp claims from the list's work queue at a time, in units of 32 for the
  // per-thread classes (0 = default)
  int shape_qpw[CQG_NLIST] = {0};
  // kernel form of a list whose class has both: 0 = per-thread (default), 1 = warp-cooperative
  int shape_var[CQG_NLIST] = {0};
  // 0: one launch per class list; 1 or 2: the lists of that tier's classes go through one
  // class-fused persistent kernel (eri_fused.cu); set by the autotuner or cqg_set_fusion
  int fused_tier = 0;
  double fusion_ms[3] = {0.0, 0.0, 0.0};   // autotuner's times of the three forms (ms)
  DevBuf<unsigned long long> d_qhead;  // work-queue head counter of every work list, then the fused one
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
  DevBuf<double> d_M, d_Mmax, d_Mpair;
  DevBuf<int> d_flags;
  DevBuf<long long> d_cnt, d_off, d_range;
  DevBuf<unsigned char> d_scan_tmp;
  DevBuf<uint2> d_qlist;
  DevBuf<double> d_G, d_X, d_AX, d_Gscratch;
  BlockTable bt;                      // the active table (bt_pair or bt_group)
  int ntask = 0;
  BlockTable bt_pair, bt_group;       // pair tasks everywhere / bra-group tasks for the sibling classes
  int ntask_pair = 0, ntask_group = 0;
  // sibling groups (Pairs): on = the sibling classes get sibling-entry lists
  int siblings = 0;
  // grouped classes: smallest number of member quartets of a pair of groups that makes a
  // sibling entry (smaller ones become pair entries); set from the sibling form's size
  int sibling_min[CQG_NQC] = {0};
  std::vector<int> pair_gsz, glead;
  std::vector<double> pair_Qc, gQ;
  int gc_beg[CQG_NPC + 1] = {0};      // first group of each pair class
  long long group_prim_pairs = 0;
  DevBuf<int> d_molgbk, d_gsz, d_gpoff, d_gnp, d_gwoff, d_glead;
  DevBuf<double> d_pair_Qc, d_gQ, d_gw;
  DevBuf<PrimPair> d_gprim;
  DevBuf<unsigned short> d_qmask;     // member masks, parallel to d_qlist
  // survivor-mask cache of the screening passes (MaskCache): steps, head, per-task slots
  DevBuf<uint2> d_masks;
  DevBuf<unsigned long long> d_mhead;
  DevBuf<long long> d_mslot;
  long long mask_steps_used = 0;      // steps the last count pass asked for
  cudaEvent_t ev[4 + 2 * CQG_NQC + 2];
  bool events = false;
  cqg_stats stats;
  double *oe_table = nullptr;   // device address of the fixed charge table (cqg_one_e_noalloc)
};

static inline Pairs make_pairs(cqg_ctx *ctx);
static inline Shells make_shells(cqg_ctx *ctx);

// classes evaluated by the warp-cooperative kernel (same rule as gen_eri.WARP_CLASSES)
__host__ __device__ constexpr bool is_warp_class(int la, int lb, int lc, int ld) {
  return ncart_c(la) * ncart_c(lb) * ncart_c(lc) * ncart_c(ld) > 150 || la + lb + lc + ld >= 6;
}

// Per-thread classes whose live state overflows one thread's 255 registers (their
// generated code spills to local memory): they also get the warp-cooperative kernel, and
// the autotuner times both forms on the class's list and keeps the faster one.
__host__ __device__ constexpr bool is_variant_class(int la, int lb, int lc, int ld) {
  const int k = ((la * 4 + lb) * 4 + lc) * 4 + ld;
  return !is_warp_class(la, lb, lc, ld) &&
         (k == ((1 * 4 + 1) * 4 + 1) * 4 + 1 || k == ((2 * 4 + 0) * 4 + 1) * 4 + 1 ||   // (pp|pp), (ds|pp)
          k == ((2 * 4 + 0) * 4 + 2) * 4 + 0 || k == ((2 * 4 + 1) * 4 + 1) * 4 + 0 ||   // (ds|ds), (dp|ps)
          k == ((2 * 4 + 1) * 4 + 2) * 4 + 0 || k == ((2 * 4 + 2) * 4 + 0) * 4 + 0 ||   // (dp|ds), (dd|ss)
          k == ((2 * 4 + 2) * 4 + 1) * 4 + 0 || k == ((3 * 4 + 0) * 4 + 1) * 4 + 0 ||   // (dd|ps), (fs|ps)
          k == ((3 * 4 + 0) * 4 + 1) * 4 + 1 || k == ((3 * 4 + 0) * 4 + 2) * 4 + 0 ||   // (fs|pp), (fs|ds)
          k == ((3 * 4 + 1) * 4 + 1) * 4 + 0 || k == ((3 * 4 + 2) * 4 + 0) * 4 + 0);    // (fp|ps), (fd|ss)
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
  const int qpw = (!SCHWARZ && ctx->shape_qpw[blk] > 0) ? ctx->shape_qpw[blk] : 1;
  k_eri_jk_warp<LA, LB, LC, LD, SCHWARZ, T><<<blocks, 32 * wpb, smem, st>>>(ctx->d_qlist.p, ctx->d_range.p, blk, sbeg,
                                                                       send, make_pairs(ctx), make_shells(ctx),
                                                                       ctx->d_boys.p, dg, Q, ctx->d_qhead.p, qpw);
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

static inline MaskCache make_mask_cache(cqg_ctx *ctx) {
  MaskCache mc;
  mc.masks = ctx->d_masks.p;
  mc.head = ctx->d_mhead.p;
  mc.slot = ctx->d_mslot.p;
  mc.cap = (long long)ctx->d_masks.n;
  return mc;
}

static inline Pairs make_pairs(cqg_ctx *ctx) {
  Pairs P;
  P.sh = ctx->d_pair_sh.p;
  P.Q = ctx->d_pair_Q.p;
  P.poff = ctx->d_pair_poff.p;
  P.np = ctx->d_pair_np.p;
  P.kk = ctx->d_pair_kk.p;
  P.prim = ctx->d_prim.p;
  P.Qc = ctx->d_pair_Qc.p;
  P.glead = ctx->d_glead.p;
  P.gQ = ctx->d_gQ.p;
  P.gsz = ctx->d_gsz.p;
  P.gpoff = ctx->d_gpoff.p;
  P.gnp = ctx->d_gnp.p;
  P.gwoff = ctx->d_gwoff.p;
  P.gprim = ctx->d_gprim.p;
  P.gw = ctx->d_gw.p;
  P.qmask = ctx->d_qmask.p;
  return P;
}
static inline Shells make_shells(cqg_ctx *ctx) {
  Shells S;
  S.center = ctx->d_center.p;
  S.bf = ctx->d_bf.p;
  S.mol = ctx->d_shmol.p;
  return S;
}
static inline Mols make_mols(cqg_ctx *ctx) {
  Mols M;
  M.nmol = ctx->nmol;
  M.shoff = ctx->d_mshoff.p;
  M.nsh = ctx->d_mnsh.p;
  M.Moff = ctx->d_mMoff.p;
  M.xoff = ctx->d_mxoff.p;
  M.nbf = ctx->d_mnbf.p;
  M.active = ctx->d_active.p;
  M.molbk = ctx->d_molbk.p;
  M.molgbk = ctx->d_molgbk.p;
  return M;
}

typedef cudaError_t (*eri_launcher)(cqg_ctx *, int blk, long long n, cudaStream_t st, const DigestGroups &dg);

// One launch of the sibling-group kernel of class (LA LB|LC LD) over list blk: CTAs of 64
// threads when the list's schedule gives 2 warps per CTA, else 128.
template <int LA, int LB, int LC, int LD, typename T>
static cudaError_t launch_gc(cqg_ctx *ctx, int blk, long long n, cudaStream_t st, const DigestGroups &dg) {
  if (n == 0) return cudaSuccess;   // n < 0: count unknown on the host (graph mode)
  const int nt = ctx->shape_wpb[blk] == 2 ? 64 : kEriThreads;
  const int cta = ctx->shape_cta[blk] > 0 ? ctx->shape_cta[blk] : 4;
  const long long cap = (long long)ctx->nsm * cta;
  const long long nb = n > 0 ? std::min<long long>((n + nt - 1) / nt, cap) : cap;
  const int chunk = 32 * (ctx->shape_qpw[blk] > 0 ? ctx->shape_qpw[blk] : 1);
  if (nt == 64)
    k_eri_gc<LA, LB, LC, LD, T, 64><<<(unsigned)nb, 64, 0, st>>>(ctx->d_qlist.p, ctx->d_range.p, blk,
                                                                make_pairs(ctx), make_shells(ctx), ctx->d_boys.p,
                                                                dg, ctx->d_qhead.p, chunk);
  else
    k_eri_gc<LA, LB, LC, LD, T, kEriThreads><<<(unsigned)nb, kEriThreads, 0, st>>>(
        ctx->d_qlist.p, ctx->d_range.p, blk, make_pairs(ctx), make_shells(ctx), ctx->d_boys.p, dg, ctx->d_qhead.p,
        chunk);
  return cudaGetLastError();
}

// Class-fused schedule (eri_fused.cu): whether class (la lb|lc ld) belongs to the fused
// kernel of `tier` (1: (ss|ss) and (ps|ss), 2: every per-thread class up to (dd|dd)), and one
// launch of that kernel over the current list ranges.
bool cqg_fused_member(int tier, int la, int lb, int lc, int ld);
cudaError_t cqg_launch_fused(cqg_ctx *ctx, int tier, cudaStream_t st, const DigestGroups &dg);

template <int LA, int LB, int LC, int LD, typename T>
static cudaError_t launch_eri(cqg_ctx *ctx, int blk, long long n, cudaStream_t st, const DigestGroups &dg) {
  if (n == 0) return cudaSuccess;   // n < 0: count unknown on the host (graph mode)
  if constexpr (is_warp_class(LA, LB, LC, LD)) {
    return launch_warp<LA, LB, LC, LD, false, T>(ctx, blk, n, 0, 0, st, dg, nullptr);
  } else {
    if constexpr (is_variant_class(LA, LB, LC, LD)) {
      if (ctx->shape_var[blk] == 1) return launch_warp<LA, LB, LC, LD, false, T>(ctx, blk, n, 0, 0, st, dg, nullptr);
    }
    const int cta = ctx->shape_cta[blk] > 0 ? ctx->shape_cta[blk] : 12;
    const long long cap = (long long)ctx->nsm * cta;
    long long nb = n > 0 ? std::min<long long>((n + kEriThreads - 1) / kEriThreads, cap) : cap;
    const int chunk = 32 * (ctx->shape_qpw[blk] > 0 ? ctx->shape_qpw[blk] : 1);
    constexpr int mb = EriMinBlocks<LA, LB, LC, LD>::v;
    if constexpr (mb > 0)
      k_eri_jk_mb<LA, LB, LC, LD, T, mb><<<(unsigned)nb, kEriThreads, 0, st>>>(
          ctx->d_qlist.p, ctx->d_range.p, blk, make_pairs(ctx), make_shells(ctx), ctx->d_boys.p, dg, ctx->d_qhead.p,
          chunk);
    else
      k_eri_jk<LA, LB, LC, LD, T><<<(unsigned)nb, kEriThreads, 0, st>>>(ctx->d_qlist.p, ctx->d_range.p, blk,
                                                                     make_pairs(ctx), make_shells(ctx),
                                                                     ctx->d_boys.p, dg, ctx->d_qhead.p, chunk);
    return cudaGetLastError();
  }
}

