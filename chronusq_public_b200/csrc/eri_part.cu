// One share of the quartet-class kernels: the launchers -- and with them the per-thread,
// warp-cooperative and sibling-group kernel instantiations -- of the classes k with
// k % CQG_NPART == CQG_PART.
// The build compiles this file CQG_NPART times, once per share, in parallel; engine.cu
// merges the shares' tables into one launcher table per precision.
#include "engine_impl.cuh"

#ifndef CQG_PART
#error "compile with -DCQG_PART=<share index>"
#endif

namespace {
constexpr int pair_index(int la, int lb) { return la * (la + 1) / 2 + lb; }
// class index in CQG_CLASS_LIST order: bra pair class i >= ket pair class j, k = i(i+1)/2 + j
constexpr int class_index(int la, int lb, int lc, int ld) {
  return pair_index(la, lb) * (pair_index(la, lb) + 1) / 2 + pair_index(lc, ld);
}
template <int A, int B, int C, int D, typename T>
constexpr eri_launcher share_launcher() {
  if constexpr (class_index(A, B, C, D) % CQG_NPART == CQG_PART) return &launch_eri<A, B, C, D, T>;
  else return nullptr;
}
#define QC(a, b, c, d, T) share_launcher<a, b, c, d, T>()
const eri_launcher kShare64[CQG_NQC] = CQG_CLASS_LIST(QC, double);
const eri_launcher kShare32[CQG_NQC] = CQG_CLASS_LIST(QC, float);
#undef QC
// sibling-group kernels of the sibling classes in this share (null for the other classes)
template <int A, int B, int C, int D, typename T>
constexpr eri_launcher share_gc_launcher() {
  if constexpr (EriGroup<A, B, C, D>::ok && class_index(A, B, C, D) % CQG_NPART == CQG_PART)
    return &launch_gc<A, B, C, D, T>;
  else
    return nullptr;
}
#define GC(a, b, c, d, T) share_gc_launcher<a, b, c, d, T>()
const eri_launcher kShareGc64[CQG_NQC] = CQG_CLASS_LIST(GC, double);
const eri_launcher kShareGc32[CQG_NQC] = CQG_CLASS_LIST(GC, float);
#undef GC
}  // namespace

#define CQG_CAT2(a, b) a##b
#define CQG_CAT(a, b) CQG_CAT2(a, b)
const eri_launcher *CQG_CAT(cqg_eri_part_table_, CQG_PART)(int fp32) { return fp32 ? kShare32 : kShare64; }
const eri_launcher *CQG_CAT(cqg_eri_part_gc_table_, CQG_PART)(int fp32) { return fp32 ? kShareGc32 : kShareGc64; }
