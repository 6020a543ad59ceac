// Shared device-side definitions for the two-electron engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// One primitive pair of a shell pair (Gaussian product theorem data).
//   p = alpha_a + alpha_b, P = (alpha_a A + alpha_b B) / p,
//   K = c_a c_b exp(-alpha_a alpha_b / p |A-B|^2)   (normalised contraction coefficients)
struct __align__(16) PrimPair {
  double p, K, Px, Py, Pz, pad;
};

#define TWO_PI_2P5 34.986836655249725   // 2 pi^(5/2)

// Boys function F_m(T), m = 0..L, in FP64.
//  T <  BOYS_TMAX: 8th-order Taylor expansion of F_L about the nearest tabulated point
//                 (grid step 0.1, F_{n}'(T) = -F_{n+1}(T)), then downward recursion
//                 F_m = (2T F_{m+1} + e^-T) / (2m+1).
//  T >= BOYS_TMAX: F_0 = sqrt(pi/T)/2 (erf(sqrt T) = 1 to 2e-17 there), then upward
//                 recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T).
// Table layout: tab[i * BOYS_NORD + n] = F_n(0.1 i), i = 0..BOYS_NT-1.
#define BOYS_TMAX 36.0
#define BOYS_NT 361
#define BOYS_NORD 32
#define BOYS_NTAYLOR 8

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
      const double e = exp(-T);
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0 / (2 * m + 1));
    }
  } else {
    F[0] = 0.5 * sqrt(3.141592653589793 / T);
    if (L > 0) {
      const double e = exp(-T);
      const double i2t = 0.5 / T;
#pragma unroll
      for (int m = 0; m < L; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * i2t;
    }
  }
}

template <int LA, int LB, int LC, int LD>
struct EriClass;
