// One persistent kernel for a set of per-thread quartet classes, fed by one device work
// queue (the class-fused schedule of the class kernels).
//
// The lists of the set's classes (FP64 and FP32 lists, heaviest class first) are laid end
// to end in one index space, each padded to whole chunks of kFusedChunk quartets.  A CTA
// claims one chunk at a time with an atomic add on a single head counter and evaluates it
// with the class's generated per-thread code and digest (eri_jk_one); so CTAs that finish
// one class go on with the next class's chunks without a kernel boundary, and the only
// tail is the end of the whole queue.  All threads of a CTA work on the same chunk, so the
// CTA re-stages its shared-memory Boys rows (one total angular momentum L at a time) only
// when a claim moves to a class of another L.  The head counter is zeroed before the
// launch; the list ranges are read on the device, so the launch needs no host round trip
// and can be captured in a CUDA graph.
//
// Two class sets ("tiers"), each its own kernel because a kernel's register allocation is
// that of its largest class:
//   tier 1: (ss|ss) and (ps|ss), the two classes that fit 128 registers (4 CTAs of 128
//           threads per SM, the occupancy of their own kernels);
//   tier 2: every per-thread class up to (dd|dd), at 255 registers.
// The autotuner times both tiers against the per-class launches and keeps the fastest.
#include "engine_impl.cuh"

namespace {

constexpr int kFusedChunk = 4 * kEriThreads;   // quartets per claim (four per thread)

// Class K of a tier's queue order (heaviest first: the longest claims are handed out while
// the queue is long).
template <int TIER, int K>
struct TierClass {
  static constexpr bool ok = false;
  static constexpr int la = 0, lb = 0, lc = 0, ld = 0;
};
#define CQG_TIER_CLASS(T, K, A, B, C, D)              \
  template <>                                         \
  struct TierClass<T, K> {                            \
    static constexpr bool ok = true;                  \
    static constexpr int la = A, lb = B, lc = C, ld = D; \
  };
CQG_TIER_CLASS(1, 0, 1, 0, 0, 0) CQG_TIER_CLASS(1, 1, 0, 0, 0, 0)
CQG_TIER_CLASS(2, 0, 2, 2, 1, 0) CQG_TIER_CLASS(2, 1, 2, 1, 2, 0) CQG_TIER_CLASS(2, 2, 2, 2, 0, 0)
CQG_TIER_CLASS(2, 3, 1, 1, 1, 1) CQG_TIER_CLASS(2, 4, 2, 1, 1, 0) CQG_TIER_CLASS(2, 5, 2, 0, 2, 0)
CQG_TIER_CLASS(2, 6, 2, 0, 1, 1) CQG_TIER_CLASS(2, 7, 2, 1, 0, 0) CQG_TIER_CLASS(2, 8, 1, 1, 1, 0)
CQG_TIER_CLASS(2, 9, 2, 0, 1, 0) CQG_TIER_CLASS(2, 10, 2, 0, 0, 0) CQG_TIER_CLASS(2, 11, 1, 1, 0, 0)
CQG_TIER_CLASS(2, 12, 1, 0, 1, 0) CQG_TIER_CLASS(2, 13, 1, 0, 0, 0) CQG_TIER_CLASS(2, 14, 0, 0, 0, 0)
#undef CQG_TIER_CLASS
constexpr int kNT1 = 2, kNT2 = 15;
constexpr int kMaxSlots = 2 * kNT2;            // FP64 and FP32 list of each class

__host__ __device__ constexpr int pair_index(int la, int lb) { return la * (la + 1) / 2 + lb; }
__host__ __device__ constexpr int class_index(int la, int lb, int lc, int ld) {
  return pair_index(la, lb) * (pair_index(la, lb) + 1) / 2 + pair_index(lc, ld);
}
template <int TIER, int K>
__host__ __device__ constexpr int tier_index() {
  using C = TierClass<TIER, K>;
  return C::ok ? class_index(C::la, C::lb, C::lc, C::ld) : -1;
}
// index (in CQG_CLASS_LIST order) of the tier's class c
template <int TIER>
__device__ __forceinline__ int tier_class_index(int c) {
  switch (c) {
#define CQG_TI(K) \
  case K: return tier_index<TIER, K>();
    CQG_TI(0) CQG_TI(1) CQG_TI(2) CQG_TI(3) CQG_TI(4) CQG_TI(5) CQG_TI(6) CQG_TI(7) CQG_TI(8) CQG_TI(9)
    CQG_TI(10) CQG_TI(11) CQG_TI(12) CQG_TI(13) CQG_TI(14)
#undef CQG_TI
  }
  return -1;
}

// Evaluate quartets [cfirst, cend) of one list with the class's per-thread code: thread t
// takes cfirst + t, cfirst + t + blockDim.x, ... (warps stay contiguous in the list, as in
// the per-class kernel).
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void fused_chunk(const uint2 *__restrict__ ql, long long cfirst, long long cend,
                                            const Pairs &P, const Shells &S, const double *boys,
                                            const DigestGroups &dg) {
  const int lane = threadIdx.x & 31;
  for (long long wfirst = cfirst + (threadIdx.x & ~31); wfirst < cend; wfirst += blockDim.x)
    eri_jk_one<LA, LB, LC, LD, T>(ql, wfirst + lane, wfirst, cend, P, S, boys, dg);
}

template <int L>
__device__ __forceinline__ void restage(int &staged, const double *boys_g, double *boys) {
  if (staged == L) return;   // block-uniform: every thread tracks the same sequence of claims
  __syncthreads();
  stage_boys<L>(boys_g, boys);
  __syncthreads();
  staged = L;
}

template <int TIER>
__global__ void __launch_bounds__(kEriThreads, TIER == 1 ? 4 : 2)
    k_eri_fused(const uint2 *__restrict__ ql, const long long *__restrict__ range, Pairs P, Shells S,
                const double *__restrict__ boys_g, DigestGroups dg, unsigned long long *__restrict__ head) {
  __shared__ __align__(16) double boys[BOYS_NT * BOYS_SROW];
  __shared__ long long s_beg[kMaxSlots], s_end[kMaxSlots], s_start[kMaxSlots + 1];
  __shared__ unsigned long long s_claim;
  constexpr int NC = TIER == 1 ? kNT1 : kNT2;
  // slot s < NC: FP64 list of the tier's class s; slot NC + s: its FP32 list
  if (threadIdx.x < 2 * NC) {
    const int s = threadIdx.x;
    const int vb = (s < NC ? 0 : CQG_NQC) + tier_class_index<TIER>(s % NC);
    s_beg[s] = range[2 * vb];
    s_end[s] = range[2 * vb + 1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long o = 0;
    for (int s = 0; s < 2 * NC; ++s) {
      s_start[s] = o;
      const long long n = s_end[s] - s_beg[s];
      o += (n + kFusedChunk - 1) / kFusedChunk * kFusedChunk;
    }
    s_start[2 * NC] = o;
  }
  __syncthreads();
  int staged = -1;
  for (;;) {
    if (threadIdx.x == 0) s_claim = atomicAdd(head, (unsigned long long)kFusedChunk);
    __syncthreads();
    const long long c0 = (long long)s_claim;
    __syncthreads();   // s_claim is rewritten by the next claim
    if (c0 >= s_start[2 * NC]) return;
    int s = 0;
    while (s_start[s + 1] <= c0) ++s;
    const long long cfirst = s_beg[s] + (c0 - s_start[s]);
    const long long cend = min(cfirst + (long long)kFusedChunk, s_end[s]);
    const bool fp32 = s >= NC;
    switch (s % NC) {   // block-uniform
#define CQG_FUSED_CASE(K)                                                                           \
  case K:                                                                                           \
    if constexpr (TierClass<TIER, K>::ok) {                                                         \
      using C = TierClass<TIER, K>;                                                                 \
      restage<C::la + C::lb + C::lc + C::ld>(staged, boys_g, boys);                                 \
      if (fp32) fused_chunk<C::la, C::lb, C::lc, C::ld, float>(ql, cfirst, cend, P, S, boys, dg);    \
      else fused_chunk<C::la, C::lb, C::lc, C::ld, double>(ql, cfirst, cend, P, S, boys, dg);        \
    }                                                                                               \
    break;
      CQG_FUSED_CASE(0) CQG_FUSED_CASE(1) CQG_FUSED_CASE(2) CQG_FUSED_CASE(3) CQG_FUSED_CASE(4)
      CQG_FUSED_CASE(5) CQG_FUSED_CASE(6) CQG_FUSED_CASE(7) CQG_FUSED_CASE(8) CQG_FUSED_CASE(9)
      CQG_FUSED_CASE(10) CQG_FUSED_CASE(11) CQG_FUSED_CASE(12) CQG_FUSED_CASE(13) CQG_FUSED_CASE(14)
#undef CQG_FUSED_CASE
      default:
        break;
    }
  }
}

}  // namespace

// Whether class (la lb|lc ld) is in the fused kernel of `tier` (1 or 2).
bool cqg_fused_member(int tier, int la, int lb, int lc, int ld) {
  static const int t1[kNT1][4] = {{1, 0, 0, 0}, {0, 0, 0, 0}};
  if (tier == 1) {
    for (const auto &c : t1)
      if (c[0] == la && c[1] == lb && c[2] == lc && c[3] == ld) return true;
    return false;
  }
  // tier 2: every per-thread class with all four angular momenta at most 2
  return tier == 2 && !is_warp_class(la, lb, lc, ld) && la <= 2 && lb <= 2 && lc <= 2 && ld <= 2;
}

// One launch of the fused kernel of `tier` over the current list ranges (d_range); the
// head counter d_qhead[CQG_NLIST] is zeroed on the stream first.
cudaError_t cqg_launch_fused(cqg_ctx *ctx, int tier, cudaStream_t st, const DigestGroups &dg) {
  cudaError_t e = cudaMemsetAsync(ctx->d_qhead.p + CQG_NLIST, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const int per_sm = tier == 1 ? 4 : 2;
  const unsigned blocks = (unsigned)(ctx->nsm * per_sm);
  if (tier == 1)
    k_eri_fused<1><<<blocks, kEriThreads, 0, st>>>(ctx->d_qlist.p, ctx->d_range.p, make_pairs(ctx), make_shells(ctx),
                                                   ctx->d_boys.p, dg, ctx->d_qhead.p + CQG_NLIST);
  else
    k_eri_fused<2><<<blocks, kEriThreads, 0, st>>>(ctx->d_qlist.p, ctx->d_range.p, make_pairs(ctx), make_shells(ctx),
                                                   ctx->d_boys.p, dg, ctx->d_qhead.p + CQG_NLIST);
  return cudaGetLastError();
}
