/*
 * CPU ORACLE (test infrastructure only) for the direct-SCF two-electron contraction.
 *
 * This file restates, in plain C, the arithmetic of the reference's hot path so the
 * CUDA engine can be checked against it.  It is linked only by the test suite, the
 * smoke check and the CPU-baseline leg of the benchmark; the product never calls it.
 *
 * What it restates (paths within the ChronusQ tree):
 *   - AOIntegrals::newTwoEContractDirect   include/aointegrals/aointegrals_contract.h:24-194
 *       quartet loop (:96-109), density-weighted Schwarz screen (:112-131),
 *       degeneracy (:133-136), J/K digest (:145-171), 0.5*scale reduction (:189-193)
 *   - AOIntegrals::computeSchwartz          src/aointegrals/aointegrals_builders.cpp:469-517
 *   - BasisSet::computeShBlkNorm            include/basisset.h:495-509
 *   - one-electron S, T, V (OneEDriver)     src/aointegrals/aointegrals_builders.cpp:27-133
 * The ERIs themselves come, in the reference, from the third-party Libint 2.2.0-alpha
 * (Engine::compute, contract.h:138-143), which is not vendored.  They are restated here
 * with the published Obara-Saika vertical recursion (Obara & Saika, JCP 84, 3963
 * (1986)) and the Head-Gordon-Pople horizontal recursion (JCP 89, 5777 (1988)), with
 * no primitive screening.  Boys values use a long-double series with downward recursion,
 * and erf plus upward recursion for large T.  Pure (L>1) shells use unit-normalised real
 * solid harmonics (Helgaker, Jorgensen, Olsen eqs. 6.4.47-50), ordered m=-l..l; the
 * transformation matrices are passed in by the caller.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAXL 4                 /* up to g shells */
#define OR_MAXLAB (2 * OR_MAXL)
#define OR_MAXM (4 * OR_MAXL + 1)

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
static int ncart_upto(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }
/* global index of a Cartesian triple in the order  L=0 | L=1 | ... , CCA within L */
static int cidx(int lx, int ly, int lz) {
  int L = lx + ly + lz;
  int i = L - lx;
  return ncart_upto(L - 1) + i * (i + 1) / 2 + lz;
}

/* ------------------------------------------------------------------ Boys ---- */
void oracle_boys(int mmax, double T, double *F) {
  if (T < 0) T = 0;
  if (T < 60.0) {
    /* F_mmax(T) = e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) */
    long double t = (long double)T;
    long double term = 1.0L / (2 * mmax + 1), sum = term;
    for (int k = 1; k < 400; k++) {
      term *= 2.0L * t / (2 * mmax + 2 * k + 1);
      sum += term;
      if (term < sum * 1e-21L) break;
    }
    long double ex = expl(-t);
    long double f = ex * sum;
    F[mmax] = (double)f;
    for (int m = mmax - 1; m >= 0; m--) {
      f = (2.0L * t * f + ex) / (2 * m + 1);
      F[m] = (double)f;
    }
  } else {
    long double t = (long double)T;
    long double ex = expl(-t);
    long double f = 0.5L * sqrtl(3.14159265358979323846264338327950288L / t) * erfl(sqrtl(t));
    F[0] = (double)f;
    for (int m = 0; m < mmax; m++) {
      f = ((2 * m + 1) * f - ex) / (2.0L * t);
      F[m + 1] = (double)f;
    }
  }
}

/* ------------------------------------------------------------ basis view ---- */
typedef struct {
  int nshell;
  const int *L, *pure, *nprim;
  const double *alpha, *coef, *centers;
  int *poff;   /* primitive offset per shell */
  int *bfoff;  /* mapSh2Bf */
  int *size;   /* functions per shell */
  int nbf;
  const double *sph[OR_MAXL + 1]; /* (2l+1) x ncart(l) row-major, may be NULL for l<2 */
} obasis;

static void obasis_init(obasis *b, int nshell, const int *L, const int *pure, const int *nprim,
                        const double *alpha, const double *coef, const double *centers,
                        const double *const *sph) {
  b->nshell = nshell; b->L = L; b->pure = pure; b->nprim = nprim;
  b->alpha = alpha; b->coef = coef; b->centers = centers;
  b->poff = (int *)malloc(sizeof(int) * nshell);
  b->bfoff = (int *)malloc(sizeof(int) * nshell);
  b->size = (int *)malloc(sizeof(int) * nshell);
  int p = 0, f = 0;
  for (int s = 0; s < nshell; s++) {
    b->poff[s] = p; p += nprim[s];
    b->size[s] = pure[s] ? 2 * L[s] + 1 : ncart(L[s]);
    b->bfoff[s] = f; f += b->size[s];
  }
  b->nbf = f;
  for (int l = 0; l <= OR_MAXL; l++) b->sph[l] = sph ? sph[l] : NULL;
}
static void obasis_free(obasis *b) { free(b->poff); free(b->bfoff); free(b->size); }

/* transform index position `pos` (stride `stride`, count `nc` Cartesian) of a block in
 * place-to-out:  out[.., m, ..] = sum_k C[m,k] in[.., k, ..].  Generic strided helper. */
static void sph_transform_axis(const double *in, double *out, int nouter, int nc, int ninner,
                               const double *C, int ns) {
  for (int o = 0; o < nouter; o++)
    for (int m = 0; m < ns; m++)
      for (int i = 0; i < ninner; i++) {
        double s = 0;
        for (int k = 0; k < nc; k++) s += C[m * nc + k] * in[(o * nc + k) * ninner + i];
        out[(o * ns + m) * ninner + i] = s;
      }
}

/* ------------------------------------------------------------------ ERI ---- */
typedef struct {
  double *V;     /* VRR table [e][f][m] */
  double *V0;    /* contracted [e][f] */
  double *T1, *T2, *cart;
  double *buf;
} eri_ws;

#define NCU(l) ((l + 1) * (l + 2) * (l + 3) / 6)
static eri_ws *eri_ws_new(void) {
  eri_ws *w = (eri_ws *)malloc(sizeof(eri_ws));
  int ne = NCU(OR_MAXLAB);
  w->V = (double *)malloc(sizeof(double) * ne * ne * OR_MAXM);
  w->V0 = (double *)malloc(sizeof(double) * ne * ne);
  int big = ne * ne * 16;
  w->T1 = (double *)malloc(sizeof(double) * big);
  w->T2 = (double *)malloc(sizeof(double) * big);
  w->cart = (double *)malloc(sizeof(double) * big);
  w->buf = (double *)malloc(sizeof(double) * big);
  return w;
}
static void eri_ws_free(eri_ws *w) {
  free(w->V); free(w->V0); free(w->T1); free(w->T2); free(w->cart); free(w->buf); free(w);
}

static const double PI = 3.14159265358979323846;

/* contracted Cartesian (ab|cd) -> w->cart[a][b][c][d] (CCA order), Cartesian sizes */
static void eri_cart(const obasis *B, int s1, int s2, int s3, int s4, eri_ws *w) {
  int la = B->L[s1], lb = B->L[s2], lc = B->L[s3], ld = B->L[s4];
  int Lab = la + lb, Lcd = lc + ld, Lt = Lab + Lcd;
  int ne = NCU(Lab), nf = NCU(Lcd);
  const double *A = B->centers + 3 * s1, *Bc = B->centers + 3 * s2;
  const double *C = B->centers + 3 * s3, *D = B->centers + 3 * s4;
  double AB2 = 0, CD2 = 0, AB[3], CD[3];
  for (int i = 0; i < 3; i++) {
    AB[i] = A[i] - Bc[i]; CD[i] = C[i] - D[i];
    AB2 += AB[i] * AB[i]; CD2 += CD[i] * CD[i];
  }
  int nm = Lt + 1;
  double *V = w->V, *V0 = w->V0;
  memset(V0, 0, sizeof(double) * ne * nf);
#define VI(e, f, m) V[((size_t)(e) * nf + (f)) * nm + (m)]
  for (int i = 0; i < B->nprim[s1]; i++)
  for (int j = 0; j < B->nprim[s2]; j++) {
    double a = B->alpha[B->poff[s1] + i], b = B->alpha[B->poff[s2] + j];
    double ca = B->coef[B->poff[s1] + i], cb = B->coef[B->poff[s2] + j];
    double zeta = a + b, P[3];
    for (int x = 0; x < 3; x++) P[x] = (a * A[x] + b * Bc[x]) / zeta;
    double Kab = exp(-a * b / zeta * AB2) * ca * cb;
    for (int k = 0; k < B->nprim[s3]; k++)
    for (int l = 0; l < B->nprim[s4]; l++) {
      double c = B->alpha[B->poff[s3] + k], d = B->alpha[B->poff[s4] + l];
      double cc = B->coef[B->poff[s3] + k], cd = B->coef[B->poff[s4] + l];
      double eta = c + d, Q[3], W[3], PQ2 = 0;
      for (int x = 0; x < 3; x++) Q[x] = (c * C[x] + d * D[x]) / eta;
      double Kcd = exp(-c * d / eta * CD2) * cc * cd;
      double rho = zeta * eta / (zeta + eta);
      for (int x = 0; x < 3; x++) {
        W[x] = (zeta * P[x] + eta * Q[x]) / (zeta + eta);
        PQ2 += (P[x] - Q[x]) * (P[x] - Q[x]);
      }
      double Fm[OR_MAXM + 1];
      oracle_boys(Lt, rho * PQ2, Fm);
      double pref = 2.0 * pow(PI, 2.5) / (zeta * eta * sqrt(zeta + eta)) * Kab * Kcd;
      for (int m = 0; m <= Lt; m++) VI(0, 0, m) = pref * Fm[m];
      /* bra VRR: [e0|00]^(m) */
      for (int L = 1; L <= Lab; L++)
        for (int ii = 0; ii <= L; ii++) {
          int ex = L - ii;
          for (int jj = 0; jj <= ii; jj++) {
            int ey = ii - jj, ez = jj;
            int e[3] = {ex, ey, ez}, dir = ex > 0 ? 0 : (ey > 0 ? 1 : 2);
            int am[3] = {ex, ey, ez}; am[dir]--;
            int ia = cidx(am[0], am[1], am[2]);
            int ie = cidx(e[0], e[1], e[2]);
            double PA = P[dir] - A[dir], WP = W[dir] - P[dir];
            int ai = am[dir];
            int ia2 = -1;
            if (ai > 0) { int a2[3] = {am[0], am[1], am[2]}; a2[dir]--; ia2 = cidx(a2[0], a2[1], a2[2]); }
            for (int m = 0; m <= Lt - L; m++) {
              double v = PA * VI(ia, 0, m) + WP * VI(ia, 0, m + 1);
              if (ai > 0) v += ai / (2 * zeta) * (VI(ia2, 0, m) - rho / zeta * VI(ia2, 0, m + 1));
              VI(ie, 0, m) = v;
            }
          }
        }
      /* ket VRR: [e0|f0]^(m) */
      for (int Lf = 1; Lf <= Lcd; Lf++)
        for (int ii = 0; ii <= Lf; ii++) {
          int fx = Lf - ii;
          for (int jj = 0; jj <= ii; jj++) {
            int fy = ii - jj, fz = jj;
            int f[3] = {fx, fy, fz}, dir = fx > 0 ? 0 : (fy > 0 ? 1 : 2);
            int cm[3] = {fx, fy, fz}; cm[dir]--;
            int ic = cidx(cm[0], cm[1], cm[2]), iff = cidx(f[0], f[1], f[2]);
            int ci = cm[dir], ic2 = -1;
            if (ci > 0) { int c2[3] = {cm[0], cm[1], cm[2]}; c2[dir]--; ic2 = cidx(c2[0], c2[1], c2[2]); }
            double QC = Q[dir] - C[dir], WQ = W[dir] - Q[dir];
            for (int Le = 0; Le <= Lab; Le++)
              for (int i2 = 0; i2 <= Le; i2++)
                for (int j2 = 0; j2 <= i2; j2++) {
                  int e0 = Le - i2, e1 = i2 - j2, e2 = j2;
                  int ee[3] = {e0, e1, e2};
                  int ie = cidx(e0, e1, e2);
                  int ei = ee[dir], iem = -1;
                  if (ei > 0) { int q[3] = {e0, e1, e2}; q[dir]--; iem = cidx(q[0], q[1], q[2]); }
                  for (int m = 0; m <= Lt - Le - Lf; m++) {
                    double v = QC * VI(ie, ic, m) + WQ * VI(ie, ic, m + 1);
                    if (ci > 0) v += ci / (2 * eta) * (VI(ie, ic2, m) - rho / eta * VI(ie, ic2, m + 1));
                    if (ei > 0) v += ei / (2 * (zeta + eta)) * VI(iem, ic, m + 1);
                    VI(ie, iff, m) = v;
                  }
                }
          }
        }
      for (int e = 0; e < ne; e++)
        for (int f = 0; f < nf; f++) V0[e * nf + f] += VI(e, f, 0);
    }
  }
#undef VI
  /* bra HRR: (a b| from (e 0|, e in [la, Lab]) ; T[a][b][f] */
  /* stage k holds (a|b) for |b|=k, |a| in [la, Lab-k]; stored with a global index */
  int nea = NCU(Lab);
  double *cur = w->T1, *nxt = w->T2;
  /* cur[a][b][f] with b index in ncart(k) */
  for (int e = 0; e < nea; e++)
    for (int f = 0; f < nf; f++) cur[e * nf + f] = V0[e * nf + f];
  for (int k = 0; k < lb; k++) {
    int nbk = ncart(k), nbk1 = ncart(k + 1);
    int amax = Lab - k - 1;
    for (int La = la; La <= amax; La++)
      for (int i1 = 0; i1 <= La; i1++)
        for (int j1 = 0; j1 <= i1; j1++) {
          int a0 = La - i1, a1 = i1 - j1, a2 = j1;
          int ia = cidx(a0, a1, a2);
          for (int i2 = 0; i2 <= k + 1; i2++)
            for (int j2 = 0; j2 <= i2; j2++) {
              int b0 = k + 1 - i2, b1 = i2 - j2, b2 = j2;
              int bb[3] = {b0, b1, b2};
              int dir = b0 > 0 ? 0 : (b1 > 0 ? 1 : 2);
              int bm[3] = {b0, b1, b2}; bm[dir]--;
              int ap[3] = {a0, a1, a2}; ap[dir]++;
              int ib = i2 * (i2 + 1) / 2 + j2;
              int ibm = ((k - bm[0]) * (k - bm[0] + 1)) / 2 + bm[2];
              int iap = cidx(ap[0], ap[1], ap[2]);
              (void)bb;
              for (int f = 0; f < nf; f++)
                nxt[((size_t)ia * nbk1 + ib) * nf + f] =
                    cur[((size_t)iap * nbk + ibm) * nf + f] + AB[dir] * cur[((size_t)ia * nbk + ibm) * nf + f];
            }
        }
    double *t = cur; cur = nxt; nxt = t;
  }
  /* extract |a|=la : bra[a][b][f] */
  int nca = ncart(la), ncb = ncart(lb), ncc = ncart(lc), ncd = ncart(ld);
  double *bra = nxt; /* reuse */
  int off_la = ncart_upto(la - 1);
  for (int a = 0; a < nca; a++)
    for (int b = 0; b < ncb; b++)
      for (int f = 0; f < nf; f++) bra[(a * ncb + b) * nf + f] = cur[((size_t)(off_la + a) * ncb + b) * nf + f];
  /* ket HRR per (a,b) */
  int nab = nca * ncb;
  double *kc = w->buf, *kn = cur;
  for (int ab = 0; ab < nab; ab++) {
    for (int f = 0; f < nf; f++) kc[f] = bra[ab * nf + f];
    double *c1 = kc, *c2 = kn;
    for (int k = 0; k < ld; k++) {
      int ndk = ncart(k), ndk1 = ncart(k + 1);
      int cmax = Lcd - k - 1;
      for (int Lc = lc; Lc <= cmax; Lc++)
        for (int i1 = 0; i1 <= Lc; i1++)
          for (int j1 = 0; j1 <= i1; j1++) {
            int c0 = Lc - i1, cc1 = i1 - j1, cc2 = j1;
            int ic = cidx(c0, cc1, cc2);
            for (int i2 = 0; i2 <= k + 1; i2++)
              for (int j2 = 0; j2 <= i2; j2++) {
                int d0 = k + 1 - i2, d1 = i2 - j2, d2 = j2;
                int dir = d0 > 0 ? 0 : (d1 > 0 ? 1 : 2);
                int dm[3] = {d0, d1, d2}; dm[dir]--;
                int cp[3] = {c0, cc1, cc2}; cp[dir]++;
                int id = i2 * (i2 + 1) / 2 + j2;
                int idm = ((k - dm[0]) * (k - dm[0] + 1)) / 2 + dm[2];
                int icp = cidx(cp[0], cp[1], cp[2]);
                c2[ic * ndk1 + id] = c1[icp * ndk + idm] + CD[dir] * c1[ic * ndk + idm];
              }
          }
      double *t = c1; c1 = c2; c2 = t;
    }
    int off_lc = ncart_upto(lc - 1);
    for (int c = 0; c < ncc; c++)
      for (int d = 0; d < ncd; d++) w->cart[(ab * ncc + c) * ncd + d] = c1[(off_lc + c) * ncd + d];
  }
}

/* contracted (ab|cd) in the reference basis (spherical for pure shells), row-major
 * [n1][n2][n3][n4] into out (must hold n1*n2*n3*n4 doubles). */
static void eri_shell(const obasis *B, int s1, int s2, int s3, int s4, eri_ws *w, double *out) {
  eri_cart(B, s1, s2, s3, s4, w);
  int sh[4] = {s1, s2, s3, s4};
  int dims[4];
  for (int i = 0; i < 4; i++) dims[i] = ncart(B->L[sh[i]]);
  double *src = w->cart, *dst = w->T1;
  for (int ax = 0; ax < 4; ax++) {
    int l = B->L[sh[ax]];
    if (!B->pure[sh[ax]]) continue;
    int nouter = 1, ninner = 1;
    for (int i = 0; i < ax; i++) nouter *= dims[i];
    for (int i = ax + 1; i < 4; i++) ninner *= dims[i];
    sph_transform_axis(src, dst, nouter, dims[ax], ninner, B->sph[l], 2 * l + 1);
    dims[ax] = 2 * l + 1;
    double *t = src; src = dst; dst = (t == w->cart) ? w->T2 : t;
  }
  int n = dims[0] * dims[1] * dims[2] * dims[3];
  memcpy(out, src, sizeof(double) * n);
}

/* public: one shell quartet */
int oracle_eri_quartet(int nshell, const int *L, const int *pure, const int *nprim,
                       const double *alpha, const double *coef, const double *centers,
                       const double *const *sph, int s1, int s2, int s3, int s4, double *out) {
  obasis B; obasis_init(&B, nshell, L, pure, nprim, alpha, coef, centers, sph);
  for (int i = 0; i < nshell; i++) if (L[i] > OR_MAXL) { obasis_free(&B); return -1; }
  eri_ws *w = eri_ws_new();
  eri_shell(&B, s1, s2, s3, s4, w, out);
  eri_ws_free(w);
  obasis_free(&B);
  return 0;
}

/* public: full ERI tensor (nbf^4, [i][j][k][l]) for tiny systems */
int oracle_eri_full(int nshell, const int *L, const int *pure, const int *nprim,
                    const double *alpha, const double *coef, const double *centers,
                    const double *const *sph, double *out) {
  obasis B; obasis_init(&B, nshell, L, pure, nprim, alpha, coef, centers, sph);
  size_t n = B.nbf;
  eri_ws *w = eri_ws_new();
  double *q = (double *)malloc(sizeof(double) * 7 * 7 * 7 * 7 * 16);
  for (int s1 = 0; s1 < nshell; s1++) for (int s2 = 0; s2 < nshell; s2++)
  for (int s3 = 0; s3 < nshell; s3++) for (int s4 = 0; s4 < nshell; s4++) {
    eri_shell(&B, s1, s2, s3, s4, w, q);
    int n1 = B.size[s1], n2 = B.size[s2], n3 = B.size[s3], n4 = B.size[s4];
    for (int i = 0, ijkl = 0; i < n1; i++) for (int j = 0; j < n2; j++)
    for (int k = 0; k < n3; k++) for (int l = 0; l < n4; l++, ijkl++)
      out[(((size_t)(B.bfoff[s1] + i) * n + B.bfoff[s2] + j) * n + B.bfoff[s3] + k) * n + B.bfoff[s4] + l] = q[ijkl];
  }
  free(q); eri_ws_free(w); obasis_free(&B);
  return 0;
}

/* --------------------------------------------------------------- Schwarz ---- */
/* computeSchwartz (builders.cpp:469-517): Q(s1,s2) = sqrt(max_ij |(ij|ij)|), symmetric,
 * Q is nshell x nshell column-major (symmetric, so either order). */
void oracle_schwarz(int nshell, const int *L, const int *pure, const int *nprim,
                    const double *alpha, const double *coef, const double *centers,
                    const double *const *sph, double *Q) {
  obasis B; obasis_init(&B, nshell, L, pure, nprim, alpha, coef, centers, sph);
  memset(Q, 0, sizeof(double) * nshell * nshell);
#pragma omp parallel
  {
    eri_ws *w = eri_ws_new();
    double *q = (double *)malloc(sizeof(double) * 7 * 7 * 7 * 7 * 16);
#pragma omp for schedule(dynamic)
    for (int s1 = 0; s1 < nshell; s1++)
      for (int s2 = 0; s2 <= s1; s2++) {
        eri_shell(&B, s1, s2, s1, s2, w, q);
        int n1 = B.size[s1], n2 = B.size[s2];
        double mx = 0;
        for (int ij = 0; ij < n1 * n2; ij++) {
          double v = fabs(q[(size_t)ij * n1 * n2 + ij]);
          if (v > mx) mx = v;
        }
        Q[s1 + (size_t)s2 * nshell] = sqrt(mx);
        Q[s2 + (size_t)s1 * nshell] = sqrt(mx);
      }
    free(q); eri_ws_free(w);
  }
  obasis_free(&B);
}

/* computeShBlkNorm (basisset.h:495-509): infinity norm (max |x|) of each shell block.
 * X column-major with leading dimension ld; out nshell x nshell column-major. */
void oracle_shblk_norm(int nshell, const int *L, const int *pure, const double *X, int ld,
                       double *out) {
  int *off = (int *)malloc(sizeof(int) * nshell), *sz = (int *)malloc(sizeof(int) * nshell);
  int f = 0;
  for (int s = 0; s < nshell; s++) { off[s] = f; sz[s] = pure[s] ? 2 * L[s] + 1 : ncart(L[s]); f += sz[s]; }
  for (int s1 = 0; s1 < nshell; s1++)
    for (int s2 = 0; s2 < nshell; s2++) {
      double mx = 0;
      for (int j = 0; j < sz[s2]; j++)
        for (int i = 0; i < sz[s1]; i++) {
          double v = fabs(X[(size_t)(off[s1] + i) + (size_t)(off[s2] + j) * ld]);
          if (v > mx) mx = v;
        }
      out[s1 + (size_t)s2 * nshell] = mx;
    }
  free(off); free(sz);
}

/* ------------------------------------------------------ direct contraction ---- */
/* newTwoEContractDirect (contract.h:24-194) for real matrices.
 * X[i], AX[i]: nbf x nbf column-major with leading dimension ld.  types: 0 COULOMB,
 * 1 EXCHANGE.  Q: Schwarz matrix (nshell^2).  AX[i] += 0.5*scale[i]*sum_thread G.
 * Returns the number of quartets that passed the screen (the unit of work).
 * `nthreads` <= 0 uses the OpenMP default; the round-robin split is s1234 % nthreads
 * exactly as contract.h:107 does.  If `per_class` is non-NULL it receives the screened
 * quartet count per (la,lb,lc,ld) in shell-index orientation, indexed
 * ((la*5+lb)*5+lc)*5+ld.  s1_begin/s1_end (-1 = all) restrict the outermost shell index,
 * and s1_mod > 1 keeps only s1 with s1 % s1_mod == s1_rem: the benchmark times a large
 * workload as s1_mod such residue classes, which together make up the whole loop. */
long long oracle_twoe_contract_direct(int nshell, const int *L, const int *pure, const int *nprim,
                                      const double *alpha, const double *coef, const double *centers,
                                      const double *const *sph, const double *Q, double thresh,
                                      int nmat, const double *const *X, double *const *AX,
                                      const int *types, const double *scale, int ld, int nthreads,
                                      long long *per_class, int s1_begin, int s1_end, int s1_mod,
                                      int s1_rem) {
  obasis B; obasis_init(&B, nshell, L, pure, nprim, alpha, coef, centers, sph);
  size_t nbf = B.nbf;
  double **blk = (double **)malloc(sizeof(double *) * nmat);
  for (int i = 0; i < nmat; i++) {
    blk[i] = (double *)malloc(sizeof(double) * nshell * nshell);
    oracle_shblk_norm(nshell, L, pure, X[i], ld, blk[i]);
  }
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  double *G = (double *)calloc((size_t)nmat * nthreads * nbf * nbf, sizeof(double));
  long long total = 0;
  long long *pc = per_class ? (long long *)calloc((size_t)nthreads * 625, sizeof(long long)) : NULL;
#define SB(i, a, b) blk[i][(a) + (size_t)(b) * nshell]
#define QQ(a, b) Q[(a) + (size_t)(b) * nshell]
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    eri_ws *w = eri_ws_new();
    double *buff = (double *)malloc(sizeof(double) * 7 * 7 * 7 * 7 * 16);
    unsigned long s1234 = 0;
    if (s1_end < 0 || s1_end > nshell) s1_end = nshell;
    if (s1_begin < 0) s1_begin = 0;
    for (int s1 = 0; s1 < nshell; s1++) {
      size_t bf1_s = B.bfoff[s1]; int n1 = B.size[s1];
      if (s1 < s1_begin || s1 >= s1_end || (s1_mod > 1 && s1 % s1_mod != s1_rem)) {
        /* bounded sample: skip this s1 but keep the global counter */
        unsigned long m = (unsigned long)s1;
        s1234 += (m + 1) * (m * (m + 1) / 2) + (m + 1) * (m + 2) / 2;
        continue;
      }
      for (int s2 = 0; s2 <= s1; s2++) {
        size_t bf2_s = B.bfoff[s2]; int n2 = B.size[s2];
        for (int s3 = 0; s3 <= s1; s3++) {
          size_t bf3_s = B.bfoff[s3]; int n3 = B.size[s3];
          int s4_max = (s1 == s3) ? s2 : s3;
          for (int s4 = 0; s4 <= s4_max; s4++, s1234++) {
            if (s1234 % (unsigned long)nthreads != (unsigned long)tid) continue;
            size_t bf4_s = B.bfoff[s4]; int n4 = B.size[s4];
            double shMax = 0;
            for (int i = 0; i < nmat; i++) {
              double m = SB(i, s1, s4);
              if (SB(i, s2, s4) > m) m = SB(i, s2, s4);
              if (SB(i, s3, s4) > m) m = SB(i, s3, s4);
              if (SB(i, s1, s3) > m) m = SB(i, s1, s3);
              if (SB(i, s2, s3) > m) m = SB(i, s2, s3);
              if (SB(i, s1, s2) > m) m = SB(i, s1, s2);
              m = m * QQ(s1, s2) * QQ(s3, s4);
              if (i == 0 || m > shMax) shMax = m;
            }
            if (shMax < thresh) continue;
            total++;
            if (pc) pc[tid * 625 + ((L[s1] * 5 + L[s2]) * 5 + L[s3]) * 5 + L[s4]]++;
            double s12_deg = (s1 == s2) ? 1.0 : 2.0;
            double s34_deg = (s3 == s4) ? 1.0 : 2.0;
            double s12_34_deg = (s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0;
            double deg = s12_deg * s34_deg * s12_34_deg;
            eri_shell(&B, s1, s2, s3, s4, w, buff);
            for (int im = 0; im < nmat; im++) {
              double *g = G + ((size_t)im * nthreads + tid) * nbf * nbf;
              const double *x = X[im];
#define GG(a, b) g[(a) + (size_t)(b) * nbf]
#define XX(a, b) x[(a) + (size_t)(b) * ld]
              if (scale[im] == 0.0) continue;
              size_t ijkl = 0;
              for (int i = 0; i < n1; i++) {
                size_t bf1 = bf1_s + i;
                for (int j = 0; j < n2; j++) {
                  size_t bf2 = bf2_s + j;
                  for (int k = 0; k < n3; k++) {
                    size_t bf3 = bf3_s + k;
                    for (int l = 0; l < n4; l++, ijkl++) {
                      size_t bf4 = bf4_s + l;
                      double v = buff[ijkl] * deg;
                      if (types[im] == 0) {
                        GG(bf1, bf2) += XX(bf4, bf3) * v;
                        GG(bf3, bf4) += XX(bf2, bf1) * v;
                        GG(bf2, bf1) += XX(bf3, bf4) * v;
                        GG(bf4, bf3) += XX(bf1, bf2) * v;
                      } else {
                        GG(bf1, bf3) += 0.5 * XX(bf2, bf4) * v;
                        GG(bf2, bf4) += 0.5 * XX(bf1, bf3) * v;
                        GG(bf1, bf4) += 0.5 * XX(bf2, bf3) * v;
                        GG(bf2, bf3) += 0.5 * XX(bf1, bf4) * v;
                        GG(bf3, bf1) += 0.5 * XX(bf4, bf2) * v;
                        GG(bf4, bf2) += 0.5 * XX(bf3, bf1) * v;
                        GG(bf4, bf1) += 0.5 * XX(bf3, bf2) * v;
                        GG(bf3, bf2) += 0.5 * XX(bf4, bf1) * v;
                      }
                    }
                  }
                }
              }
#undef GG
#undef XX
            }
          }
        }
      }
    }
    free(buff);
    eri_ws_free(w);
  }
  for (int im = 0; im < nmat; im++)
    for (int t = 0; t < nthreads; t++) {
      const double *g = G + ((size_t)im * nthreads + t) * nbf * nbf;
      for (size_t c = 0; c < nbf; c++)
        for (size_t r = 0; r < nbf; r++) AX[im][r + c * ld] += 0.5 * scale[im] * g[r + c * nbf];
    }
  if (pc) {
    for (int k = 0; k < 625; k++) {
      long long s = 0;
      for (int t = 0; t < nthreads; t++) s += pc[t * 625 + k];
      per_class[k] = s;
    }
    free(pc);
  }
#undef SB
#undef QQ
  free(G);
  for (int i = 0; i < nmat; i++) free(blk[i]);
  free(blk);
  obasis_free(&B);
  return total;
}

/* --------------------------------------------------------- one-electron ---- */
/* 1D Obara-Saika overlap table S[i][j], i<=imax, j<=jmax (without the 3D prefactor) */
static void os_overlap_1d(double PA, double PB, double p, int imax, int jmax, double *S, int ldS) {
  S[0] = 1.0;
  for (int i = 0; i <= imax; i++)
    for (int j = 0; j <= jmax; j++) {
      if (i == 0 && j == 0) continue;
      double v;
      if (i > 0) {
        v = PA * S[(i - 1) * ldS + j];
        if (i > 1) v += (i - 1) / (2 * p) * S[(i - 2) * ldS + j];
        if (j > 0) v += j / (2 * p) * S[(i - 1) * ldS + j - 1];
      } else {
        v = PB * S[i * ldS + j - 1];
        if (j > 1) v += (j - 1) / (2 * p) * S[i * ldS + j - 2];
      }
      S[i * ldS + j] = v;
    }
}

/* S, T (kinetic) and V (nuclear attraction of point charges Zc at Rc) in the reference
 * basis; each nbf x nbf column-major. */
void oracle_one_e(int nshell, const int *L, const int *pure, const int *nprim,
                  const double *alpha, const double *coef, const double *centers,
                  const double *const *sph, int ncharge, const double *Zc, const double *Rc,
                  double *S, double *T, double *V) {
  obasis B; obasis_init(&B, nshell, L, pure, nprim, alpha, coef, centers, sph);
  size_t nbf = B.nbf;
#pragma omp parallel for schedule(dynamic)
  for (int s1 = 0; s1 < nshell; s1++)
    for (int s2 = 0; s2 < nshell; s2++) {
      int la = L[s1], lb = L[s2], nca = ncart(la), ncb = ncart(lb);
      double Sc[256], Tc[256], Vc[256];
      memset(Sc, 0, sizeof(Sc)); memset(Tc, 0, sizeof(Tc)); memset(Vc, 0, sizeof(Vc));
      const double *A = centers + 3 * s1, *Bc = centers + 3 * s2;
      double AB[3], AB2 = 0;
      for (int x = 0; x < 3; x++) { AB[x] = A[x] - Bc[x]; AB2 += AB[x] * AB[x]; }
      for (int i = 0; i < nprim[s1]; i++)
        for (int j = 0; j < nprim[s2]; j++) {
          double a = alpha[B.poff[s1] + i], b = alpha[B.poff[s2] + j];
          double ca = coef[B.poff[s1] + i], cb = coef[B.poff[s2] + j];
          double p = a + b, P[3];
          for (int x = 0; x < 3; x++) P[x] = (a * A[x] + b * Bc[x]) / p;
          double K = exp(-a * b / p * AB2) * ca * cb;
          double pre = K * pow(PI / p, 1.5);
          double S1[3][8 * 8];
          for (int x = 0; x < 3; x++) os_overlap_1d(P[x] - A[x], P[x] - Bc[x], p, la + 1, lb + 2, S1[x], 8);
          /* overlap + kinetic */
          for (int ia = 0; ia < nca; ia++) {
            int ax[3] = {0, 0, 0}; { int ii = 0, c = 0; for (int i1 = 0; i1 <= la; i1++) for (int j1 = 0; j1 <= i1; j1++, c++) if (c == ia) { ax[0] = la - i1; ax[1] = i1 - j1; ax[2] = j1; ii = 1; } (void)ii; }
            for (int ib = 0; ib < ncb; ib++) {
              int bx[3] = {0, 0, 0}; { int c = 0; for (int i1 = 0; i1 <= lb; i1++) for (int j1 = 0; j1 <= i1; j1++, c++) if (c == ib) { bx[0] = lb - i1; bx[1] = i1 - j1; bx[2] = j1; } }
              double s[3], t[3];
              for (int x = 0; x < 3; x++) {
                int ii = ax[x], jj = bx[x];
                s[x] = S1[x][ii * 8 + jj];
                double tk = -2.0 * b * b * S1[x][ii * 8 + jj + 2] + b * (2 * jj + 1) * S1[x][ii * 8 + jj];
                if (jj >= 2) tk -= 0.5 * jj * (jj - 1) * S1[x][ii * 8 + jj - 2];
                t[x] = tk;
              }
              Sc[ia * ncb + ib] += pre * s[0] * s[1] * s[2];
              Tc[ia * ncb + ib] += pre * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2]);
            }
          }
          /* nuclear attraction: OS VRR on the bra (e|0)^(m) then HRR */
          int Lab = la + lb;
          double VV[165 * 9];
          for (int cI = 0; cI < ncharge; cI++) {
            const double *C = Rc + 3 * cI;
            double PC2 = 0, PA[3], PCv[3];
            for (int x = 0; x < 3; x++) { PA[x] = P[x] - A[x]; PCv[x] = P[x] - C[x]; PC2 += PCv[x] * PCv[x]; }
            double Fm[16];
            oracle_boys(Lab, p * PC2, Fm);
            double base = -Zc[cI] * 2.0 * PI / p * K;
            int nm = Lab + 1;
            for (int m = 0; m <= Lab; m++) VV[m] = base * Fm[m];
            for (int Le = 1; Le <= Lab; Le++)
              for (int i1 = 0; i1 <= Le; i1++)
                for (int j1 = 0; j1 <= i1; j1++) {
                  int e[3] = {Le - i1, i1 - j1, j1};
                  int dir = e[0] > 0 ? 0 : (e[1] > 0 ? 1 : 2);
                  int am[3] = {e[0], e[1], e[2]}; am[dir]--;
                  int ia = cidx(am[0], am[1], am[2]), ie = cidx(e[0], e[1], e[2]);
                  int ai = am[dir], ia2 = -1;
                  if (ai > 0) { int q[3] = {am[0], am[1], am[2]}; q[dir]--; ia2 = cidx(q[0], q[1], q[2]); }
                  for (int m = 0; m <= Lab - Le; m++) {
                    double v = PA[dir] * VV[ia * nm + m] - PCv[dir] * VV[ia * nm + m + 1];
                    if (ai > 0) v += ai / (2 * p) * (VV[ia2 * nm + m] - VV[ia2 * nm + m + 1]);
                    VV[ie * nm + m] = v;
                  }
                }
            /* HRR (a|b+1_i) = (a+1_i|b) + AB_i (a|b) */
            double H1[165 * 15], H2[165 * 15];
            int ne = NCU(Lab);
            for (int e = 0; e < ne; e++) H1[e] = VV[e * nm];
            double *cur = H1, *nxt = H2;
            for (int k = 0; k < lb; k++) {
              int nbk = ncart(k), nbk1 = ncart(k + 1);
              for (int La = la; La <= Lab - k - 1; La++)
                for (int i1 = 0; i1 <= La; i1++)
                  for (int j1 = 0; j1 <= i1; j1++) {
                    int a0 = La - i1, a1 = i1 - j1, a2 = j1;
                    int iaa = cidx(a0, a1, a2);
                    for (int i2 = 0; i2 <= k + 1; i2++)
                      for (int j2 = 0; j2 <= i2; j2++) {
                        int bb[3] = {k + 1 - i2, i2 - j2, j2};
                        int dir = bb[0] > 0 ? 0 : (bb[1] > 0 ? 1 : 2);
                        int bm[3] = {bb[0], bb[1], bb[2]}; bm[dir]--;
                        int ap[3] = {a0, a1, a2}; ap[dir]++;
                        int ib = i2 * (i2 + 1) / 2 + j2;
                        int ibm = ((k - bm[0]) * (k - bm[0] + 1)) / 2 + bm[2];
                        nxt[iaa * nbk1 + ib] = cur[cidx(ap[0], ap[1], ap[2]) * nbk + ibm] + AB[dir] * cur[iaa * nbk + ibm];
                      }
                  }
              double *tt = cur; cur = nxt; nxt = tt;
            }
            int off = ncart_upto(la - 1);
            for (int ia = 0; ia < nca; ia++)
              for (int ib = 0; ib < ncb; ib++) Vc[ia * ncb + ib] += cur[(off + ia) * ncb + ib];
          }
        }
      /* spherical transform and store */
      double *blocks[3] = {Sc, Tc, Vc};
      double *outs[3] = {S, T, V};
      for (int q = 0; q < 3; q++) {
        double tmp[256], tmp2[256];
        int d0 = nca, d1 = ncb;
        memcpy(tmp, blocks[q], sizeof(double) * nca * ncb);
        if (pure[s1]) { sph_transform_axis(tmp, tmp2, 1, nca, d1, B.sph[la], 2 * la + 1); d0 = 2 * la + 1; memcpy(tmp, tmp2, sizeof(double) * d0 * d1); }
        if (pure[s2]) { sph_transform_axis(tmp, tmp2, d0, ncb, 1, B.sph[lb], 2 * lb + 1); d1 = 2 * lb + 1; memcpy(tmp, tmp2, sizeof(double) * d0 * d1); }
        for (int i = 0; i < d0; i++)
          for (int j = 0; j < d1; j++) outs[q][(B.bfoff[s1] + i) + (size_t)(B.bfoff[s2] + j) * nbf] = tmp[i * d1 + j];
      }
    }
  obasis_free(&B);
}

/* Electric dipole integrals <a| r_k - O_k |b>, k = x, y, z, about origin O, in the
 * reference basis (each nbf x nbf column-major).  The reference takes them from Libint's
 * first electric multipole operator (AOIntegrals::elecDipole_, split per component in
 * AOIntegrals::breakUpMultipole, src/aointegrals/aointegrals_builders.cpp:640-650).  Here:
 * the 1D Obara-Saika overlap table and x - O_x = (x - B_x) + (B_x - O_x), so the x factor is
 * S(i, j+1) + (B_x - O_x) S(i, j). */
void oracle_dipole(int nshell, const int *L, const int *pure, const int *nprim,
                   const double *alpha, const double *coef, const double *centers,
                   const double *const *sph, const double *origin, double *Dx, double *Dy, double *Dz) {
  obasis B; obasis_init(&B, nshell, L, pure, nprim, alpha, coef, centers, sph);
  size_t nbf = B.nbf;
  double *outs[3] = {Dx, Dy, Dz};
#pragma omp parallel for schedule(dynamic)
  for (int s1 = 0; s1 < nshell; s1++)
    for (int s2 = 0; s2 < nshell; s2++) {
      int la = L[s1], lb = L[s2], nca = ncart(la), ncb = ncart(lb);
      double Mc[3][256];
      memset(Mc, 0, sizeof(Mc));
      const double *A = centers + 3 * s1, *Bc = centers + 3 * s2;
      double AB2 = 0;
      for (int x = 0; x < 3; x++) AB2 += (A[x] - Bc[x]) * (A[x] - Bc[x]);
      for (int i = 0; i < nprim[s1]; i++)
        for (int j = 0; j < nprim[s2]; j++) {
          double a = alpha[B.poff[s1] + i], b = alpha[B.poff[s2] + j];
          double ca = coef[B.poff[s1] + i], cb = coef[B.poff[s2] + j];
          double p = a + b, P[3];
          for (int x = 0; x < 3; x++) P[x] = (a * A[x] + b * Bc[x]) / p;
          double pre = exp(-a * b / p * AB2) * ca * cb * pow(PI / p, 1.5);
          double S1[3][8 * 8];
          for (int x = 0; x < 3; x++) os_overlap_1d(P[x] - A[x], P[x] - Bc[x], p, la + 1, lb + 2, S1[x], 8);
          for (int ia = 0; ia < nca; ia++) {
            int ax[3] = {0, 0, 0};
            { int c = 0; for (int i1 = 0; i1 <= la; i1++) for (int j1 = 0; j1 <= i1; j1++, c++) if (c == ia) { ax[0] = la - i1; ax[1] = i1 - j1; ax[2] = j1; } }
            for (int ib = 0; ib < ncb; ib++) {
              int bx[3] = {0, 0, 0};
              { int c = 0; for (int i1 = 0; i1 <= lb; i1++) for (int j1 = 0; j1 <= i1; j1++, c++) if (c == ib) { bx[0] = lb - i1; bx[1] = i1 - j1; bx[2] = j1; } }
              double s[3], d[3];
              for (int x = 0; x < 3; x++) {
                s[x] = S1[x][ax[x] * 8 + bx[x]];
                d[x] = S1[x][ax[x] * 8 + bx[x] + 1] + (Bc[x] - origin[x]) * s[x];
              }
              Mc[0][ia * ncb + ib] += pre * d[0] * s[1] * s[2];
              Mc[1][ia * ncb + ib] += pre * s[0] * d[1] * s[2];
              Mc[2][ia * ncb + ib] += pre * s[0] * s[1] * d[2];
            }
          }
        }
      for (int q = 0; q < 3; q++) {
        double tmp[256], tmp2[256];
        int d0 = nca, d1 = ncb;
        memcpy(tmp, Mc[q], sizeof(double) * nca * ncb);
        if (pure[s1]) { sph_transform_axis(tmp, tmp2, 1, nca, d1, B.sph[la], 2 * la + 1); d0 = 2 * la + 1; memcpy(tmp, tmp2, sizeof(double) * d0 * d1); }
        if (pure[s2]) { sph_transform_axis(tmp, tmp2, d0, ncb, 1, B.sph[lb], 2 * lb + 1); d1 = 2 * lb + 1; memcpy(tmp, tmp2, sizeof(double) * d0 * d1); }
        for (int i = 0; i < d0; i++)
          for (int j = 0; j < d1; j++) outs[q][(B.bfoff[s1] + i) + (size_t)(B.bfoff[s2] + j) * nbf] = tmp[i * d1 + j];
      }
    }
  obasis_free(&B);
}
