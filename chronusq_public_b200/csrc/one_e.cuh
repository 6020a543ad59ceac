// One-electron integrals S, T, V on the device (the reference computes them on the host
// with Libint's OneEDriver, src/aointegrals/aointegrals_builders.cpp:27-133, 337-467).
//
// McMurchie-Davidson, one thread per shell pair (a >= b):
//   S_ab  = sum_prims K (pi/p)^(3/2) Ex^{ax bx}_0 Ey^{ay by}_0 Ez^{az bz}_0
//   T_ab  = sum over directions of T1D_x S1D_y S1D_z with
//           T1D_ij = -2 b^2 S1D_{i,j+2} + b (2j+1) S1D_{ij} - j(j-1)/2 S1D_{i,j-2}
//   V_ab  = -sum_C Z_C (2 pi/p) K sum_tuv E^{ab}_{tuv} R_{tuv}(p, P - C)
// with K = c_a c_b exp(-a b/p |A-B|^2), S1D_ij = E^{ij}_0 sqrt(pi/p), then the Cartesian
// blocks are transformed to real solid harmonics for pure (L > 1) shells.
#pragma once
#include "eri_common.cuh"

#define OE_MAXL 3
#define OE_NT (2 * OE_MAXL + 3)   // t range of E[i][j][t] with j up to lb + 2

struct OneEShells {
  const int *L, *nprim, *poff, *bf;
  const double *alpha, *coef;
  const double3 *center;
};

// 1D E[i][j][t] for i <= la, j <= lbp (lbp = lb + 2), t <= i + j
__device__ __forceinline__ void oe_build_E(double E[OE_MAXL + 1][OE_MAXL + 3][OE_NT], int la, int lbp, double PA,
                                           double PB, double o2p) {
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lbp; ++j)
      for (int t = 0; t < OE_NT; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = 1.0;
  for (int j = 1; j <= lbp; ++j)
    for (int t = 0; t <= j; ++t) {
      double v = PB * E[0][j - 1][t];
      if (t > 0) v += o2p * E[0][j - 1][t - 1];
      if (t + 1 <= j - 1) v += (t + 1) * E[0][j - 1][t + 1];
      E[0][j][t] = v;
    }
  for (int i = 1; i <= la; ++i)
    for (int j = 0; j <= lbp; ++j)
      for (int t = 0; t <= i + j; ++t) {
        double v = PA * E[i - 1][j][t];
        if (t > 0) v += o2p * E[i - 1][j][t - 1];
        if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
        E[i][j][t] = v;
      }
}

__device__ __forceinline__ void oe_cart(int l, int k, int &x, int &y, int &z) {
  int i = 0;
  while ((i + 1) * (i + 2) / 2 <= k) ++i;
  const int j = k - i * (i + 1) / 2;
  x = l - i;
  y = i - j;
  z = j;
}

__device__ __forceinline__ int oe_hidx(int t, int u, int v) {
  const int n = t + u + v, i = n - t;
  return (n * (n + 1) * (n + 2)) / 6 + (i * (i + 1)) / 2 + v;
}

// runtime-L Boys from the global table (layout of eri_common.cuh)
__device__ __forceinline__ void boys_eval_rt(int L, double T, const double *__restrict__ tab, double *F) {
  if (T < BOYS_TMAX) {
    const int i = __double2int_rn(T * 10.0);
    const double x = (double)i * 0.1 - T;
    const double *row = tab + i * BOYS_NORD + L;
    double f = row[BOYS_NTAYLOR];
    for (int k = BOYS_NTAYLOR; k >= 1; --k) f = row[k - 1] + x * f / k;
    F[L] = f;
    const double e = exp(-T);
    for (int m = L - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + e) / (2 * m + 1);
  } else {
    F[0] = 0.5 * sqrt(3.141592653589793 / T);
    const double e = exp(-T);
    for (int m = 0; m < L; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

// Molecule layout for batches: shell -> molecule, per-molecule output offset / leading
// dimension and charge range.  For one molecule: xoff = 0, ld = caller's, all charges.
struct OneEMols {
  const int *shmol;
  const long long *xoff;
  const int *nbf;
  const int *coff;   // charges of molecule m: [coff[m], coff[m+1])
  int batch;
};

__global__ void k_one_e(OneEShells sh, const int2 *__restrict__ pairs, long long npairs, int ncharge,
                        const double *__restrict__ Zc, const double3 *__restrict__ Rc,
                        const double *__restrict__ boys, double *S0, double *T0, double *V0, int ld, OneEMols om) {
  const long long ip = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ip >= npairs) return;
  const int a = pairs[ip].x, b = pairs[ip].y;
  double *S = S0, *T = T0, *V = V0;
  int c_beg = 0, c_end = ncharge;
  if (om.batch) {
    const int m = om.shmol[a];
    S += om.xoff[m];
    T += om.xoff[m];
    V += om.xoff[m];
    ld = om.nbf[m];
    c_beg = om.coff[m];
    c_end = om.coff[m + 1];
  }
  const int la = sh.L[a], lb = sh.L[b];
  const int nca = (la + 1) * (la + 2) / 2, ncb = (lb + 1) * (lb + 2) / 2;
  const double3 A = sh.center[a], B = sh.center[b];
  const double ABx = A.x - B.x, ABy = A.y - B.y, ABz = A.z - B.z;
  const double AB2 = ABx * ABx + ABy * ABy + ABz * ABz;
  double Sc[100], Tc[100], Vc[100];
  for (int k = 0; k < nca * ncb; ++k) Sc[k] = Tc[k] = Vc[k] = 0.0;
  double Ex[OE_MAXL + 1][OE_MAXL + 3][OE_NT], Ey[OE_MAXL + 1][OE_MAXL + 3][OE_NT], Ez[OE_MAXL + 1][OE_MAXL + 3][OE_NT];
  double R[165], Rn[165], F[2 * OE_MAXL + 1];
  const double pi = 3.141592653589793;
  for (int i = 0; i < sh.nprim[a]; ++i)
    for (int j = 0; j < sh.nprim[b]; ++j) {
      const double al = sh.alpha[sh.poff[a] + i], be = sh.alpha[sh.poff[b] + j];
      const double p = al + be, o2p = 0.5 / p;
      const double K = sh.coef[sh.poff[a] + i] * sh.coef[sh.poff[b] + j] * exp(-al * be / p * AB2);
      const double Px = (al * A.x + be * B.x) / p, Py = (al * A.y + be * B.y) / p, Pz = (al * A.z + be * B.z) / p;
      oe_build_E(Ex, la, lb + 2, Px - A.x, Px - B.x, o2p);
      oe_build_E(Ey, la, lb + 2, Py - A.y, Py - B.y, o2p);
      oe_build_E(Ez, la, lb + 2, Pz - A.z, Pz - B.z, o2p);
      const double s1 = sqrt(pi / p);
      const double pre = K * s1 * s1 * s1;
      for (int ka = 0; ka < nca; ++ka) {
        int ax, ay, az;
        oe_cart(la, ka, ax, ay, az);
        for (int kb = 0; kb < ncb; ++kb) {
          int bx, by, bz;
          oe_cart(lb, kb, bx, by, bz);
          const double sx = Ex[ax][bx][0], sy = Ey[ay][by][0], sz = Ez[az][bz][0];
          Sc[ka * ncb + kb] += pre * sx * sy * sz;
          double tx = -2.0 * be * be * Ex[ax][bx + 2][0] + be * (2 * bx + 1) * sx;
          if (bx >= 2) tx -= 0.5 * bx * (bx - 1) * Ex[ax][bx - 2][0];
          double ty = -2.0 * be * be * Ey[ay][by + 2][0] + be * (2 * by + 1) * sy;
          if (by >= 2) ty -= 0.5 * by * (by - 1) * Ey[ay][by - 2][0];
          double tz = -2.0 * be * be * Ez[az][bz + 2][0] + be * (2 * bz + 1) * sz;
          if (bz >= 2) tz -= 0.5 * bz * (bz - 1) * Ez[az][bz - 2][0];
          Tc[ka * ncb + kb] += pre * (tx * sy * sz + sx * ty * sz + sx * sy * tz);
        }
      }
      const int Lab = la + lb;
      for (int c = c_beg; c < c_end; ++c) {
        const double3 C = Rc[c];
        const double X = Px - C.x, Y = Py - C.y, Z = Pz - C.z;
        boys_eval_rt(Lab, p * (X * X + Y * Y + Z * Z), boys, F);
        // R^{(n)}_{tuv}, n = Lab .. 0
        double fac = -Zc[c] * 2.0 * pi / p * K;
        double facs[2 * OE_MAXL + 1];
        for (int n = 0; n <= Lab; ++n) {
          facs[n] = fac * F[n];
          fac *= -2.0 * p;
        }
        R[0] = facs[Lab];
        for (int n = Lab - 1; n >= 0; --n) {
          for (int tot = 0; tot <= Lab - n; ++tot)
            for (int ii = 0; ii <= tot; ++ii)
              for (int jj = 0; jj <= ii; ++jj) {
                const int t = tot - ii, u = ii - jj, v = jj;
                double val;
                if (tot == 0) val = facs[n];
                else if (t > 0) val = X * R[oe_hidx(t - 1, u, v)] + (t > 1 ? (t - 1) * R[oe_hidx(t - 2, u, v)] : 0.0);
                else if (u > 0) val = Y * R[oe_hidx(t, u - 1, v)] + (u > 1 ? (u - 1) * R[oe_hidx(t, u - 2, v)] : 0.0);
                else val = Z * R[oe_hidx(t, u, v - 1)] + (v > 1 ? (v - 1) * R[oe_hidx(t, u, v - 2)] : 0.0);
                Rn[oe_hidx(t, u, v)] = val;
              }
          for (int k = 0; k < (Lab - n + 1) * (Lab - n + 2) * (Lab - n + 3) / 6; ++k) R[k] = Rn[k];
        }
        for (int ka = 0; ka < nca; ++ka) {
          int ax, ay, az;
          oe_cart(la, ka, ax, ay, az);
          for (int kb = 0; kb < ncb; ++kb) {
            int bx, by, bz;
            oe_cart(lb, kb, bx, by, bz);
            double s = 0.0;
            for (int t = 0; t <= ax + bx; ++t)
              for (int u = 0; u <= ay + by; ++u)
                for (int v = 0; v <= az + bz; ++v) s += Ex[ax][bx][t] * Ey[ay][by][u] * Ez[az][bz][v] * R[oe_hidx(t, u, v)];
            Vc[ka * ncb + kb] += s;
          }
        }
      }
    }
  // spherical transform and store both triangles
  double *blocks[3] = {Sc, Tc, Vc};
  double *outs[3] = {S, T, V};
  const int pa = la > 1, pb = lb > 1;
  const int na = pa ? 2 * la + 1 : nca, nb = pb ? 2 * lb + 1 : ncb;
  const double *Ca = la == 2 ? kSph2 : kSph3, *Cb = lb == 2 ? kSph2 : kSph3;
  const int a0 = sh.bf[a], b0 = sh.bf[b];
  for (int q = 0; q < 3; ++q) {
    const double *M = blocks[q];
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < nb; ++j) {
        double s = 0.0;
        for (int ka = 0; ka < nca; ++ka) {
          const double ca = pa ? Ca[i * nca + ka] : (ka == i ? 1.0 : 0.0);
          if (ca == 0.0) continue;
          for (int kb = 0; kb < ncb; ++kb) {
            const double cb = pb ? Cb[j * ncb + kb] : (kb == j ? 1.0 : 0.0);
            if (cb == 0.0) continue;
            s += ca * cb * M[ka * ncb + kb];
          }
        }
        outs[q][(size_t)(a0 + i) + (size_t)(b0 + j) * ld] = s;
        outs[q][(size_t)(b0 + j) + (size_t)(a0 + i) * ld] = s;
      }
  }
}

// Electric dipole integrals <a| r_k - O_k |b> (k = x, y, z) of one shell pair, Cartesian
// blocks Dc[k][ka * ncb + kb].  McMurchie-Davidson first moment (Helgaker, Jorgensen & Olsen
// eq. 9.5.43): the x factor is sqrt(pi/p) (E^{ij}_1 + (P_x - O_x) E^{ij}_0), the y and z
// factors are overlaps.  The reference takes these from Libint's first electric multipole
// operator about the origin (AOIntegrals::elecDipoleSep_, aointegrals_builders.cpp:640-650).
__device__ __forceinline__ void oe_dipole_pair(const OneEShells &sh, int a, int b, double3 O, double Dc[3][100]) {
  const int la = sh.L[a], lb = sh.L[b];
  const int nca = (la + 1) * (la + 2) / 2, ncb = (lb + 1) * (lb + 2) / 2;
  const double3 A = sh.center[a], B = sh.center[b];
  const double ABx = A.x - B.x, ABy = A.y - B.y, ABz = A.z - B.z;
  const double AB2 = ABx * ABx + ABy * ABy + ABz * ABz;
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < nca * ncb; ++i) Dc[k][i] = 0.0;
  double Ex[OE_MAXL + 1][OE_MAXL + 3][OE_NT], Ey[OE_MAXL + 1][OE_MAXL + 3][OE_NT], Ez[OE_MAXL + 1][OE_MAXL + 3][OE_NT];
  const double pi = 3.141592653589793;
  for (int i = 0; i < sh.nprim[a]; ++i)
    for (int j = 0; j < sh.nprim[b]; ++j) {
      const double al = sh.alpha[sh.poff[a] + i], be = sh.alpha[sh.poff[b] + j];
      const double p = al + be, o2p = 0.5 / p;
      const double K = sh.coef[sh.poff[a] + i] * sh.coef[sh.poff[b] + j] * exp(-al * be / p * AB2);
      const double Px = (al * A.x + be * B.x) / p, Py = (al * A.y + be * B.y) / p, Pz = (al * A.z + be * B.z) / p;
      oe_build_E(Ex, la, lb, Px - A.x, Px - B.x, o2p);
      oe_build_E(Ey, la, lb, Py - A.y, Py - B.y, o2p);
      oe_build_E(Ez, la, lb, Pz - A.z, Pz - B.z, o2p);
      const double s1 = sqrt(pi / p);
      const double pre = K * s1 * s1 * s1;
      for (int ka = 0; ka < nca; ++ka) {
        int ax, ay, az;
        oe_cart(la, ka, ax, ay, az);
        for (int kb = 0; kb < ncb; ++kb) {
          int bx, by, bz;
          oe_cart(lb, kb, bx, by, bz);
          const double sx = Ex[ax][bx][0], sy = Ey[ay][by][0], sz = Ez[az][bz][0];
          const double mx = Ex[ax][bx][1] + (Px - O.x) * sx;
          const double my = Ey[ay][by][1] + (Py - O.y) * sy;
          const double mz = Ez[az][bz][1] + (Pz - O.z) * sz;
          Dc[0][ka * ncb + kb] += pre * mx * sy * sz;
          Dc[1][ka * ncb + kb] += pre * sx * my * sz;
          Dc[2][ka * ncb + kb] += pre * sx * sy * mz;
        }
      }
    }
}

// Cartesian block M[ka * ncb + kb] of shell pair (a, b) to real solid harmonics for pure
// (L > 1) shells, stored at rows a0.., columns b0.. of out and, transposed, at rows b0..,
// columns a0.. (column-major, leading dimension ld).
__device__ __forceinline__ void oe_store_pair(const double *M, int la, int lb, int a0, int b0, double *out, int ld) {
  const int nca = (la + 1) * (la + 2) / 2, ncb = (lb + 1) * (lb + 2) / 2;
  const int pa = la > 1, pb = lb > 1;
  const int na = pa ? 2 * la + 1 : nca, nb = pb ? 2 * lb + 1 : ncb;
  const double *Ca = la == 2 ? kSph2 : kSph3, *Cb = lb == 2 ? kSph2 : kSph3;
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      double s = 0.0;
      for (int ka = 0; ka < nca; ++ka) {
        const double ca = pa ? Ca[i * nca + ka] : (ka == i ? 1.0 : 0.0);
        if (ca == 0.0) continue;
        for (int kb = 0; kb < ncb; ++kb) {
          const double cb = pb ? Cb[j * ncb + kb] : (kb == j ? 1.0 : 0.0);
          if (cb == 0.0) continue;
          s += ca * cb * M[ka * ncb + kb];
        }
      }
      out[(size_t)(a0 + i) + (size_t)(b0 + j) * ld] = s;
      out[(size_t)(b0 + j) + (size_t)(a0 + i) * ld] = s;
    }
}

// Dipole integrals of one molecule, one thread per shell pair (a >= b); D0 holds the x, y
// and z matrices at D0, D0 + ld * nbf and D0 + 2 * ld * nbf.
__global__ void k_dipole(OneEShells sh, const int2 *__restrict__ pairs, long long npairs, double3 O, double *D0,
                         int ld, int nbf) {
  const long long ip = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (ip >= npairs) return;
  const int a = pairs[ip].x, b = pairs[ip].y;
  double Dc[3][100];
  oe_dipole_pair(sh, a, b, O, Dc);
  for (int k = 0; k < 3; ++k)
    oe_store_pair(Dc[k], sh.L[a], sh.L[b], sh.bf[a], sh.bf[b], D0 + (size_t)k * ld * nbf, ld);
}
