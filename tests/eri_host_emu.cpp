// Test infrastructure: a host (g++) build of the generated per-thread ERI code
// (csrc/gen_eri.py output, eri_classes.cuh).  The CUDA qualifiers become plain C++ and the
// few device intrinsics get host definitions, so the same generated arithmetic runs on the
// CPU and is checked against the oracle without a GPU.  Nothing in the library uses this
// file; tests/test_eri_host_emu.py compiles it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

// Compiled with an include directory whose cuda_runtime.h is empty: the definitions the
// generated code needs from it follow here.
#define __device__
#define __host__
#define __global__ static inline   // the kernels compile but are not called here
#define __forceinline__ inline
#define __constant__
#define __align__(n) alignas(n)
struct double2 {
  double x, y;
};
struct double3 {
  double x, y, z;
};
struct int2 {
  int x, y;
};
struct EmuDim {
  unsigned x;
};
// one thread per block: stage_boys fills the whole table, and a kernel body is run for
// thread index ip by setting blockIdx.x = ip
static EmuDim threadIdx = {0}, blockDim = {1}, blockIdx = {0};
static inline int __double2int_rn(double x) { return (int)std::nearbyint(x); }   // ties to even
static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
template <typename T>
static inline T __ldg(const T *p) {
  return *p;
}

#include "eri_classes.cuh"
#include "one_e.cuh"

namespace {

// Boys table in the engine's global layout (cqg_create in csrc/engine.cu):
// tab[i * BOYS_NORD + n] = F_n(0.1 i), then tab[BOYS_NT * BOYS_NORD + i] = exp(-0.1 i).
// F_nmax from its series in long double, lower orders by downward recursion.
std::vector<double> boys_table() {
  std::vector<double> tab(BOYS_TABLE_SIZE);
  for (int i = 0; i < BOYS_NT; ++i) {
    const long double T = (long double)i / 10.0L;
    const int nmax = BOYS_NORD - 1;
    long double term = 1.0L / (2 * nmax + 1), sum = term;
    for (int k = 1; k < 2000; ++k) {
      term *= 2.0L * T / (2 * nmax + 2 * k + 1);
      sum += term;
      if (term < sum * 1e-22L) break;
    }
    const long double ex = expl(-T);
    long double f = ex * sum;
    tab[i * BOYS_NORD + nmax] = (double)f;
    for (int m = nmax - 1; m >= 0; --m) {
      f = (2.0L * T * f + ex) / (2 * m + 1);
      tab[i * BOYS_NORD + m] = (double)f;
    }
    tab[BOYS_NT * BOYS_NORD + i] = (double)ex;
  }
  return tab;
}

// All primitive pairs of two shells (Gaussian product theorem data, PrimPair layout).
std::vector<PrimPair> prim_pairs(int na, const double *aa, const double *ca, const double *A, int nb,
                                 const double *ab, const double *cb, const double *B) {
  const double s2pi52 = std::sqrt(2.0 * std::pow(3.14159265358979323846, 2.5));
  double AB2 = 0;
  for (int x = 0; x < 3; ++x) AB2 += (A[x] - B[x]) * (A[x] - B[x]);
  std::vector<PrimPair> out;
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      const double al = aa[i], be = ab[j], p = al + be;
      PrimPair pp;
      pp.p = p;
      pp.ip = 1.0 / p;
      pp.Kp = s2pi52 * ca[i] * cb[j] * std::exp(-al * be / p * AB2) / p;
      pp.Px = (al * A[0] + be * B[0]) / p;
      pp.Py = (al * A[1] + be * B[1]) / p;
      pp.Pz = (al * A[2] + be * B[2]) / p;
      out.push_back(pp);
    }
  return out;
}

constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
constexpr bool warp_class(int a, int b, int c, int d) {
  return ncart(a) * ncart(b) * ncart(c) * ncart(d) > 150 || a + b + c + d >= 6;
}

struct Quartet {
  const PrimPair *bra, *ket;
  int nbra, nket;
  double3 A, B, C, D;
  double *out;
};

template <int LA, int LB, int LC, int LD, typename T>
int call(const Quartet &q) {
  if constexpr (warp_class(LA, LB, LC, LD)) {
    return -1;   // evaluated by the warp-cooperative kernel, not by generated code
  } else {
    static const std::vector<double> tab = boys_table();
    alignas(16) static double s[BOYS_NT * BOYS_SROW];
    stage_boys<LA + LB + LC + LD>(tab.data(), s);
    constexpr int n = (LA > 1 ? 2 * LA + 1 : ncart(LA)) * (LB > 1 ? 2 * LB + 1 : ncart(LB)) *
                      (LC > 1 ? 2 * LC + 1 : ncart(LC)) * (LD > 1 ? 2 * LD + 1 : ncart(LD));
    T v[n];
    EriClass<LA, LB, LC, LD>::template run<T>(q.bra, q.nbra, q.ket, q.nket, q.A, q.B, q.C, q.D, s, v);
    for (int k = 0; k < n; ++k) q.out[k] = (double)v[k];
    return n;
  }
}

template <int L>
int boys_one(double T, int sm, double *F) {
  static const std::vector<double> tab = boys_table();
  alignas(16) static double s[BOYS_NT * BOYS_SROW];
  static bool staged = false;
  if (!staged) {
    stage_boys<L>(tab.data(), s);
    staged = true;
  }
  if (sm == 1)
    boys_eval_sm<L>(T, s, F);
  else if (sm == 2)
    boys_eval_rt(L, T, tab.data(), F);
  else
    boys_eval<L>(T, tab.data(), F);
  return L + 1;
}

template <int... Ls>
int boys_dispatch(int L, double T, int sm, double *F, std::integer_sequence<int, Ls...>) {
  int r = -1;
  ((L == Ls ? (r = boys_one<Ls>(T, sm, F), 0) : 0), ...);
  return r;
}

struct Entry {
  int la, lb, lc, ld;
  int (*f64)(const Quartet &);
  int (*f32)(const Quartet &);
};
#define EMU_ENTRY(a, b, c, d, T) Entry{a, b, c, d, &call<a, b, c, d, double>, &call<a, b, c, d, float>}
const Entry kTable[] = CQG_CLASS_LIST(EMU_ENTRY, double);

}  // namespace

extern "C" {

// One contracted quartet (ab|cd) of class (la lb|lc ld), in the engine's orientation
// (la >= lb, lc >= ld, bra pair class >= ket pair class).  nprim[4]; alpha/coef: the four
// shells' exponents and normalised contraction coefficients, concatenated; centers: 4 x 3.
// out gets the spherical (L > 1) or Cartesian components, row-major [a][b][c][d].
// fp32 != 0 runs the FP32 instantiation (Boys values FP64, everything after in float).
// Returns the number of values, or -1 for a class the generated code does not cover.
int emu_eri(int la, int lb, int lc, int ld, const int *nprim, const double *alpha, const double *coef,
            const double *centers, int fp32, double *out) {
  int off[4] = {0, nprim[0], nprim[0] + nprim[1], nprim[0] + nprim[1] + nprim[2]};
  std::vector<PrimPair> bra = prim_pairs(nprim[0], alpha + off[0], coef + off[0], centers, nprim[1],
                                         alpha + off[1], coef + off[1], centers + 3);
  std::vector<PrimPair> ket = prim_pairs(nprim[2], alpha + off[2], coef + off[2], centers + 6, nprim[3],
                                         alpha + off[3], coef + off[3], centers + 9);
  Quartet q{bra.data(), ket.data(), (int)bra.size(), (int)ket.size(),
            {centers[0], centers[1], centers[2]}, {centers[3], centers[4], centers[5]},
            {centers[6], centers[7], centers[8]}, {centers[9], centers[10], centers[11]}, out};
  for (const Entry &e : kTable)
    if (e.la == la && e.lb == lb && e.lc == lc && e.ld == ld) return fp32 ? e.f32(q) : e.f64(q);
  return -1;
}

// The device Boys evaluations for total angular momentum L (0..12): boys_eval_sm on the
// shared-memory rows of stage_boys<L> (per-thread kernels) when sm == 1, boys_eval_rt
// (runtime L, one-electron kernel) when sm == 2, else boys_eval on the global table (warp
// kernels).  F gets F_0..F_L at T; returns L + 1, or -1.
int emu_boys(int L, double T, int sm, double *F) {
  return boys_dispatch(L, T, sm, F, std::make_integer_sequence<int, 13>{});
}

// The one-electron dipole device code (oe_dipole_pair + oe_store_pair of one_e.cuh) over
// every shell pair a >= b of a basis: D gets the x, y, z matrices (nbf x nbf each,
// column-major, consecutive).  bf[s] is shell s's first basis function.
void emu_dipole(int nshell, const int *L, const int *nprim, const int *poff, const int *bf, const double *alpha,
                const double *coef, const double *centers, const double *origin, int nbf, double *D) {
  std::vector<double3> cen(nshell);
  for (int s = 0; s < nshell; ++s) cen[s] = {centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]};
  OneEShells sh;
  sh.L = L;
  sh.nprim = nprim;
  sh.poff = poff;
  sh.bf = bf;
  sh.alpha = alpha;
  sh.coef = coef;
  sh.center = cen.data();
  const double3 O = {origin[0], origin[1], origin[2]};
  for (int a = 0; a < nshell; ++a)
    for (int b = 0; b <= a; ++b) {
      double Dc[3][100];
      oe_dipole_pair(sh, a, b, O, Dc);
      for (int k = 0; k < 3; ++k) oe_store_pair(Dc[k], L[a], L[b], bf[a], bf[b], D + (size_t)k * nbf * nbf, nbf);
    }
}

// The one-electron kernel body (k_one_e) run for every shell pair a >= b of one molecule:
// S, T, V (nbf x nbf each, column-major) for point charges Zc at Rc (ncharge x 3).
void emu_one_e(int nshell, const int *L, const int *nprim, const int *poff, const int *bf, const double *alpha,
               const double *coef, const double *centers, int ncharge, const double *Zc, const double *Rc, int nbf,
               double *S, double *T, double *V) {
  static const std::vector<double> tab = boys_table();
  std::vector<double3> cen(nshell), rc(ncharge);
  for (int s = 0; s < nshell; ++s) cen[s] = {centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]};
  for (int c = 0; c < ncharge; ++c) rc[c] = {Rc[3 * c], Rc[3 * c + 1], Rc[3 * c + 2]};
  std::vector<int2> pairs;
  for (int a = 0; a < nshell; ++a)
    for (int b = 0; b <= a; ++b) pairs.push_back({a, b});
  OneEShells sh;
  sh.L = L;
  sh.nprim = nprim;
  sh.poff = poff;
  sh.bf = bf;
  sh.alpha = alpha;
  sh.coef = coef;
  sh.center = cen.data();
  OneEMols om;
  std::memset(&om, 0, sizeof(om));
  for (size_t ip = 0; ip < pairs.size(); ++ip) {
    blockIdx.x = (unsigned)ip;
    k_one_e(sh, pairs.data(), (long long)pairs.size(), ncharge, Zc, rc.data(), tab.data(), S, T, V, nbf, om);
  }
  blockIdx.x = 0;
}

#ifdef EMU_MEMBERS
}  // extern "C"

#include "eri_gc_classes.cuh"

namespace {

struct MemberQuartet {
  const PrimPair *bra, *ket;
  const double *bw, *kw;
  int nbra, nket;
  double3 A, B, C, D;
  double *out;
};

template <int LA, int LB, int LC, int LD, int MB, int MK>
int call_members(const MemberQuartet &q) {
  static const std::vector<double> tab = boys_table();
  alignas(16) static double s[BOYS_NT * BOYS_SROW];
  stage_boys<LA + LB + LC + LD>(tab.data(), s);
  constexpr int n = (LA > 1 ? 2 * LA + 1 : ncart(LA)) * (LB > 1 ? 2 * LB + 1 : ncart(LB)) *
                    (LC > 1 ? 2 * LC + 1 : ncart(LC)) * (LD > 1 ? 2 * LD + 1 : ncart(LD));
  EriClassGC<LA, LB, LC, LD, MB, MK>::template run<double>(q.bra, q.bw, q.nbra, q.ket, q.kw, q.nket, q.A, q.B,
                                                           q.C, q.D, s, q.out);
  return n * MB * MK;
}

struct MemberEntry {
  int la, lb, lc, ld, mb, mk;
  int (*f)(const MemberQuartet &);
};
#define EMU_MEMBER_ENTRY(a, b, c, d, m, k) MemberEntry{a, b, c, d, m, k, &call_members<a, b, c, d, m, k>}
const MemberEntry kMemberTable[] = CQG_GC_LIST(EMU_MEMBER_ENTRY);

// Unit-coefficient primitive pairs of two shells, and each member's coefficient products
// w[m * na * nb + i * nb + j] = ca_m[i] cb_m[j] in the same (i outer, j inner) order.
std::vector<double> member_weights(int m, int na, const double *ca, int nb, const double *cb) {
  std::vector<double> w((size_t)m * na * nb);
  for (int k = 0; k < m; ++k)
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < nb; ++j) w[(size_t)k * na * nb + i * nb + j] = ca[k * na + i] * cb[k * nb + j];
  return w;
}

}  // namespace

extern "C" {

// Sibling-member quartets: mb bra pairs and mk ket pairs sharing exponents.  alpha holds
// the four shells' exponents; coef holds, in order, the a coefficients of the mb bra
// members (mb x na), then b (mb x nb), then c (mk x nc), then d (mk x nd).  out gets the
// mb * mk quartets, member (i, j) at out + (i * mk + j) * n.
int emu_eri_members(int la, int lb, int lc, int ld, int mb, int mk, const int *nprim, const double *alpha,
                    const double *coef, const double *centers, double *out) {
  const int na = nprim[0], nb = nprim[1], nc = nprim[2], nd = nprim[3];
  const double *ea = alpha, *eb = ea + na, *ec = eb + nb, *ed = ec + nc;
  const double *ca = coef, *cb = ca + mb * na, *cc = cb + mb * nb, *cd = cc + mk * nc;
  std::vector<double> one(std::max(std::max(na, nb), std::max(nc, nd)), 1.0);
  std::vector<PrimPair> bra = prim_pairs(na, ea, one.data(), centers, nb, eb, one.data(), centers + 3);
  std::vector<PrimPair> ket = prim_pairs(nc, ec, one.data(), centers + 6, nd, ed, one.data(), centers + 9);
  std::vector<double> bw = member_weights(mb, na, ca, nb, cb), kw = member_weights(mk, nc, cc, nd, cd);
  MemberQuartet q{bra.data(), ket.data(), bw.data(), kw.data(), (int)bra.size(), (int)ket.size(),
                  {centers[0], centers[1], centers[2]}, {centers[3], centers[4], centers[5]},
                  {centers[6], centers[7], centers[8]}, {centers[9], centers[10], centers[11]}, out};
  for (const MemberEntry &e : kMemberTable)
    if (e.la == la && e.lb == lb && e.lc == lc && e.ld == ld && e.mb == mb && e.mk == mk) return e.f(q);
  return -1;
}
#endif

}  // extern "C"
