// Warp-cooperative McMurchie-Davidson ERI + J/K digest for the high angular momentum
// classes, whose per-quartet intermediates do not fit in one thread's registers.
//
// One warp evaluates one shell quartet at a time.  The 32 lanes share, in shared memory:
//   Eb, Ek : 1D Hermite expansion coefficients E^{ij}_t of the bra / ket primitive pair
//   R      : R_{tuv} for t+u+v <= L (built level by level, n = L .. 0)
//   W      : W[tuv][cd] = sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi} R_{t+tau,..}
//            accumulated over ket primitive pairs (tuv over the bra Hermite set)
//   C      : C[ab][cd] = sum_{tuv} E^{ab}_{tuv} W[tuv][cd], accumulated over bra primitives
// then transform C to real solid harmonics for pure shells and digest into J and K with
// the lanes spread over the output elements.  Same mathematics as the generated
// per-thread functions (Helgaker, Jorgensen & Olsen ch. 9.9); only the work split differs.
#pragma once
#include "eri_common.cuh"

namespace warpmd {

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nherm(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }
__host__ __device__ constexpr int nfun(int l) { return l > 1 ? 2 * l + 1 : ncart(l); }

// index of Hermite / Cartesian triple (t,u,v) in the "by total, CCA within total" order
__device__ __forceinline__ int hidx(int t, int u, int v) {
  const int n = t + u + v;
  const int i = n - t;
  return (n * (n + 1) * (n + 2)) / 6 + (i * (i + 1)) / 2 + v;
}
// decode Cartesian index k of angular momentum l (CCA order) into exponents
__device__ __forceinline__ void cart_of(int l, int k, int &x, int &y, int &z) {
  int i = 0;
  while ((i + 1) * (i + 2) / 2 <= k) ++i;
  const int j = k - i * (i + 1) / 2;
  x = l - i;
  y = i - j;
  z = j;
}
__device__ __forceinline__ void herm_of(int h, int &t, int &u, int &v) {
  int n = 0;
  while (nherm(n) <= h) ++n;
  cart_of(n, h - nherm(n - 1), t, u, v);
}

// Solid-harmonic coefficient tables (rows m=-l..l over CCA Cartesians), set by the host.
struct SphTables {
  double c2[5 * 6];
  double c3[7 * 10];
};

template <int LA, int LB>
struct PairDims {
  static constexpr int NE = (LA + 1) * (LB + 1) * (LA + LB + 1);  // E[i][j][t] per direction
};

// 1D Hermite coefficients E[i][j][t], i<=la, j<=lb, t<=i+j for one direction, by lanes.
// Layout: ((i*(lb+1)) + j)*(la+lb+1) + t.  Built serially by one lane (tiny).
template <int LA, int LB, typename T>
__device__ __forceinline__ void build_E1(T *E, T PA, T PB, T o2p) {
  constexpr int NT = LA + LB + 1;
#pragma unroll
  for (int k = 0; k < (LA + 1) * (LB + 1) * NT; ++k) E[k] = T(0);
  E[0] = T(1);
  // grow j at i = 0
#pragma unroll
  for (int j = 1; j <= LB; ++j)
#pragma unroll
    for (int t = 0; t <= j; ++t) {
      const T *prev = E + (0 * (LB + 1) + (j - 1)) * NT;
      T v = PB * (t <= j - 1 ? prev[t] : T(0));
      if (t > 0) v += o2p * prev[t - 1];
      if (t + 1 <= j - 1) v += T(t + 1) * prev[t + 1];
      E[(0 * (LB + 1) + j) * NT + t] = v;
    }
#pragma unroll
  for (int i = 1; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j) {
      const T *prev = E + ((i - 1) * (LB + 1) + j) * NT;
      const int tm = i - 1 + j;
#pragma unroll
      for (int t = 0; t <= i + j; ++t) {
        T v = (t <= tm ? PA * prev[t] : T(0));
        if (t > 0 && t - 1 <= tm) v += o2p * prev[t - 1];
        if (t + 1 <= tm) v += T(t + 1) * prev[t + 1];
        E[(i * (LB + 1) + j) * NT + t] = v;
      }
    }
}

template <int L>
__device__ __forceinline__ const double *sph_rows(const SphTables &st) {
  return L == 2 ? st.c2 : st.c3;
}

// Transform axis `ax` of a 4-index block from Cartesian to spherical (pure shells).
// in: dims d[0..3] (row-major), out: same with d[ax] -> 2l+1.  Lanes over output.
template <typename T>
__device__ __forceinline__ void sph_axis(const T *in, T *out, const int *d, int ax, int l, const double *C,
                                         int lane) {
  int nout[4] = {d[0], d[1], d[2], d[3]};
  const int ns = 2 * l + 1, nc = ncart(l);
  nout[ax] = ns;
  int inner = 1;
  for (int k = ax + 1; k < 4; ++k) inner *= d[k];
  int outer = 1;
  for (int k = 0; k < ax; ++k) outer *= d[k];
  const int total = outer * ns * inner;
  for (int e = lane; e < total; e += 32) {
    const int in_i = e % inner;
    const int m = (e / inner) % ns;
    const int o = e / (inner * ns);
    T s = T(0);
    for (int k = 0; k < nc; ++k) {
      const double c = C[m * nc + k];
      if (c != 0.0) s += T(c) * in[(o * nc + k) * inner + in_i];
    }
    out[e] = s;
  }
}

template <int LA, int LB, int LC, int LD>
struct WarpDims {
  static constexpr int L = LA + LB + LC + LD;
  static constexpr int P = LA + LB, Q = LC + LD;
  static constexpr int HP = nherm(P), HL = nherm(L);
  static constexpr int NCAB = ncart(LA) * ncart(LB), NCCD = ncart(LC) * ncart(LD);
  static constexpr int NEB = (LA + 1) * (LB + 1) * (P + 1), NEK = (LC + 1) * (LD + 1) * (Q + 1);
  static constexpr int NW = HP * NCCD;
  static constexpr int NC = NCAB * NCCD;
  // shared doubles per warp: Eb[3], Ek[3], R (2 levels), W, C
  static constexpr int SMEM = 3 * NEB + 3 * NEK + 2 * HL + NW + NC;
  static constexpr int NSA = nfun(LA), NSB = nfun(LB), NSC = nfun(LC), NSD = nfun(LD);
  // staged density blocks of the digest: (d,c), (b,a), (b,d), (a,c), (b,c), (a,d)
  static constexpr int NXS = NSC * NSD + NSA * NSB + NSB * NSD + NSA * NSC + NSB * NSC + NSA * NSD;
};

}  // namespace warpmd
