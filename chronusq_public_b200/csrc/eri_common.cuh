// Shared device-side definitions for the two-electron engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// One primitive pair of a shell pair (Gaussian product theorem data).
//   p = alpha_a + alpha_b, ip = 1/p, P = (alpha_a A + alpha_b B) / p,
//   Kp = sqrt(2 pi^(5/2)) c_a c_b exp(-alpha_a alpha_b / p |A-B|^2) / p
// so that the primitive-quartet prefactor 2 pi^(5/2) K_ab K_cd / (p q sqrt(p+q)) is
// Kp_ab * Kp_cd * rsqrt(p+q)  (c_a, c_b: normalised contraction coefficients).
struct __align__(16) PrimPair {
  double p, Kp, Px, Py, Pz, ip;
};

#define TWO_PI_2P5 34.986836655249725   // 2 pi^(5/2)

// Boys function F_m(T), m = 0..L, in FP64.
//  T <  BOYS_TMAX: 8th-order Taylor expansion of F_L about the nearest tabulated point
//                 (grid step 0.1, F_{n}'(T) = -F_{n+1}(T)), then downward recursion
//                 F_m = (2T F_{m+1} + e^-T) / (2m+1).
//  T >= BOYS_TMAX: F_0 = sqrt(pi/T)/2 (erf(sqrt T) = 1 to 2e-17 there), then upward
//                 recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T); T^(-1/2) from rsqrt.
// Table layout: tab[i * BOYS_NORD + n] = F_n(0.1 i), i = 0..BOYS_NT-1, followed by
// tab[BOYS_NT * BOYS_NORD + i] = exp(-0.1 i).
#define BOYS_TMAX 36.0
#define BOYS_NT 361
#define BOYS_NORD 32
#define BOYS_NTAYLOR 8
#define BOYS_TABLE_SIZE (BOYS_NT * BOYS_NORD + BOYS_NT)

// e^x for |x| <= 0.05 from its degree-9 Taylor polynomial (remainder < 3e-20 relative).
__device__ __forceinline__ double exp_small(double x) {
  double ex = 1.0 / 362880.0;
  ex = fma(x, ex, 1.0 / 40320.0);
  ex = fma(x, ex, 1.0 / 5040.0);
  ex = fma(x, ex, 1.0 / 720.0);
  ex = fma(x, ex, 1.0 / 120.0);
  ex = fma(x, ex, 1.0 / 24.0);
  ex = fma(x, ex, 1.0 / 6.0);
  ex = fma(x, ex, 0.5);
  ex = fma(x, ex, 1.0);
  return fma(x, ex, 1.0);
}

template <int L>
__device__ __forceinline__ void boys_eval(double T, const double* __restrict__ tab, double* F) {
  if (T < BOYS_TMAX) {
    const int i = __double2int_rn(T * 10.0);
    const double x = (double)i * 0.1 - T;   // -(T - T_i)
    const double* row = tab + i * BOYS_NORD + L;
    double f = __ldg(row + BOYS_NTAYLOR);
#pragma unroll
    for (int k = BOYS_NTAYLOR; k >= 1; --k) f = __ldg(row + k - 1) + x * f * (1.0 / k);
    F[L] = f;
    if (L > 0) {
      const double e = __ldg(tab + BOYS_NT * BOYS_NORD + i) * exp_small(x);
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0 / (2 * m + 1));
    }
  } else {
    // F_0 = (sqrt(pi) / 2) T^(-1/2) and 1 / (2T) from one reciprocal square root
    const double r = rsqrt(T);
    F[0] = 0.88622692545275801 * r;
    if (L > 0) {
      const double e = exp(-T);
      const double i2t = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < L; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * i2t;
    }
  }
}

// Shared-memory copy of the rows a kernel of total angular momentum L needs, with the
// Taylor coefficients already divided by k! and e^{-T_i} appended (16-byte aligned rows,
// read as five double2):
//   s[i * BOYS_SROW + k] = F_{L+k}(0.1 i) / k!,  k = 0..BOYS_NTAYLOR
//   s[i * BOYS_SROW + BOYS_NTAYLOR + 1] = exp(-0.1 i)
#define BOYS_SROW (BOYS_NTAYLOR + 2)
template <int L>
__device__ __forceinline__ void stage_boys(const double *__restrict__ tab, double *s) {
  for (int k = threadIdx.x; k < BOYS_NT * BOYS_SROW; k += blockDim.x) {
    const int i = k / BOYS_SROW, c = k % BOYS_SROW;
    if (c <= BOYS_NTAYLOR) {
      double inv_fact = 1.0;
      for (int j = 2; j <= c; ++j) inv_fact /= (double)j;
      s[k] = __ldg(tab + i * BOYS_NORD + L + c) * inv_fact;
    } else {
      s[k] = exp(-0.1 * (double)i);
    }
  }
}

// boys_eval with the table staged in shared memory (layout of stage_boys<L>).  Below
// BOYS_TMAX, e^{-T} = e^{-T_i} e^{x} with x = T_i - T, |x| <= 0.05, from the degree-9
// Taylor polynomial of e^x (remainder < 3e-20 relative), instead of a call to exp().
template <int L>
__device__ __forceinline__ void boys_eval_sm(double T, const double *s, double *F) {
  static_assert(BOYS_NTAYLOR == 8 && BOYS_SROW == 10, "row layout read as five double2");
  if (T < BOYS_TMAX) {
    const int i = __double2int_rn(T * 10.0);
    const double x = (double)i * 0.1 - T;
    const double2 *row = reinterpret_cast<const double2 *>(s + i * BOYS_SROW);
    const double2 c01 = row[0], c23 = row[1], c45 = row[2], c67 = row[3], c8e = row[4];
    double f = c8e.x;
    f = fma(x, f, c67.y);
    f = fma(x, f, c67.x);
    f = fma(x, f, c45.y);
    f = fma(x, f, c45.x);
    f = fma(x, f, c23.y);
    f = fma(x, f, c23.x);
    f = fma(x, f, c01.y);
    f = fma(x, f, c01.x);
    F[L] = f;
    if (L > 0) {
      const double e = c8e.y * exp_small(x);
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0 / (2 * m + 1));
    }
  } else {
    // F_0 = (sqrt(pi) / 2) T^(-1/2) and 1 / (2T) from one reciprocal square root
    const double r = rsqrt(T);
    F[0] = 0.88622692545275801 * r;
    if (L > 0) {
      // F_1 = (F_0 - e^-T) / (2T): for T >= 36, e^-T / F_0 < 1.6e-15, within the Taylor
      // branch's accuracy, so L = 1 drops it; higher orders need it
      const double e = L == 1 ? 0.0 : exp(-T);
      const double i2t = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < L; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * i2t;
    }
  }
}

template <int LA, int LB, int LC, int LD>
struct EriClass;
