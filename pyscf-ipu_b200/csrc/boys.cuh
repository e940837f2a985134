// Boys function F_m(T) = int_0^1 u^{2m} exp(-T u^2) du for the ERI kernels.
//
// T < B2_BOYS_TMAX: Taylor expansion of F_L around the nearest tabulated point T_k = k*dT
//   (dF_m/dT = -F_{m+1}), then downward recursion F_m = (2T F_{m+1} + e^{-T}) / (2m+1),
//   which is stable.  The table holds F_0..F_{B2_BOYS_NM-1} at every T_k and is filled on
//   the host in double precision by the convergent series
//   F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)).
// T >= B2_BOYS_TMAX: F_0 = sqrt(pi/T)/2 (erf(sqrt T) = 1 to double precision) and upward
//   recursion F_{m+1} = ((2m+1) F_m - e^{-T}) / (2T), stable for large T.
#pragma once
#include "common.cuh"

#define B2_BOYS_DT 0.125
#define B2_BOYS_INV_DT 8.0
#define B2_BOYS_TMAX 40.0
#define B2_BOYS_NT 322          // T_k = k*DT, k = 0..321 (covers TMAX + DT/2)
#define B2_BOYS_NM 14           // m = 0..13 (L <= 4 plus 9 Taylor terms)

// host: fill table[k*NM + m]
static void b2_boys_fill_table(double *table) {
  for (int k = 0; k < B2_BOYS_NT; ++k) {
    double t = k * B2_BOYS_DT;
    int mmax = B2_BOYS_NM - 1;
    double term = 1.0 / (2 * mmax + 1), sum = term;
    for (int j = 1; j < 2000; ++j) {
      term *= 2.0 * t / (2 * mmax + 2 * j + 1);
      sum += term;
      if (term < 1e-20 * sum) break;
    }
    double et = exp(-t);
    double f[B2_BOYS_NM];
    f[mmax] = et * sum;
    for (int m = mmax - 1; m >= 0; --m) f[m] = (2.0 * t * f[m + 1] + et) / (2 * m + 1);
    for (int m = 0; m < B2_BOYS_NM; ++m) table[k * B2_BOYS_NM + m] = f[m];
  }
}

template <typename T> struct B2BoysTerms;
template <> struct B2BoysTerms<double> { static constexpr int n = 9; };
template <> struct B2BoysTerms<float> { static constexpr int n = 5; };   // remainder < 1e-8

// e^{-t}: exact for float64; hardware 2^x for float32 (t < 40: relative error < 1e-6 times
// a term that the downward recursion adds to F values of order >= e^{-t})
template <typename T> B2_HD T b2_exp_neg(T t) { return exp(-t); }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ float b2_exp_neg<float>(float t) { return __expf(-t); }
#endif

// 1 / t and 1 / sqrt(t): exact for float64; for float32 one hardware reciprocal square root
// (relative error ~1e-7) and its square
template <typename T> B2_HD void b2_inv_rsqrt(T t, T &inv, T &rt) { inv = (T)1 / t; rt = sqrt(inv); }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ void b2_inv_rsqrt<float>(float t, float &inv, float &rt) {
  rt = rsqrtf(t);
  inv = rt * rt;
}
#endif

// float32 F_0 alone (the (ss|ss) class) from the error function instead of the table:
// F_0(T) = sqrt(pi)/2 erf(sqrt T) / sqrt T, one hardware reciprocal square root and erff
// (relative error a few 1e-7, like the table path) and no table reads
template <typename T> struct B2BoysErfF0 { static constexpr bool value = false; };
template <> struct B2BoysErfF0<float> { static constexpr bool value = true; };

// F[0..L] at T; `table` is the table in double (float64 kernels) or float (float32 kernels).
template <typename T, int L, typename TT>
B2_HD void b2_boys(T t, const TT *__restrict__ table, T *F) {
  if constexpr (L == 0 && B2BoysErfF0<T>::value) {
    if (t < (T)1e-6) {                                // F_0 = 1 - T/3 + T^2/10 - ...
      F[0] = (T)1 - t * (T)(1.0 / 3.0);
    } else {
      T inv, rt;                                      // 1 / T, 1 / sqrt(T)
      b2_inv_rsqrt<T>(t, inv, rt);
      F[0] = (T)0.886226925452758014 * rt * erf(t * rt);
    }
    return;
  }
  if (t < (T)B2_BOYS_TMAX) {
    int k = (int)(t * (T)B2_BOYS_INV_DT + (T)0.5);
    T dt = (T)(k * B2_BOYS_DT) - t;           // T_k - T
    const TT *row = table + k * B2_BOYS_NM + L;
    constexpr int NT = B2BoysTerms<T>::n;
    // Horner: sum_j F_{L+j}(T_k) dt^j / j!
    T acc = (T)row[NT - 1];
#pragma unroll
    for (int j = NT - 1; j >= 1; --j) acc = (T)row[j - 1] + acc * dt * (T)(1.0 / j);
    F[L] = acc;
    if (L > 0) {
      T et = b2_exp_neg<T>(t);
      T t2 = t + t;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + et) * (T)(1.0 / (2 * m + 1));
    }
  } else {
    T inv, rt;                                        // 1 / T, 1 / sqrt(T)
    b2_inv_rsqrt<T>(t, inv, rt);
    F[0] = (T)0.886226925452758014 * rt;              // sqrt(pi)/2 / sqrt(T)
#pragma unroll
    for (int m = 0; m < L; ++m) F[m + 1] = (T)(2 * m + 1) * (T)0.5 * inv * F[m];
  }
}

// reciprocal / inverse square root: exact for float64, fast hardware forms for float32
template <typename T> B2_HD T b2_div(T a, T b) { return a / b; }
template <typename T> B2_HD T b2_rsqrt(T x) { return (T)1 / sqrt(x); }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ float b2_div<float>(float a, float b) { return __fdividef(a, b); }
template <> __device__ __forceinline__ float b2_rsqrt<float>(float x) { return rsqrtf(x); }
#endif
// a / s and 1 / sqrt(s): exact for float64; for float32 one hardware reciprocal square root r
// and a / s = a r^2 (no separate division)
template <typename T> B2_HD void b2_rho_rs(T a, T s, T &q, T &rs) { q = b2_div<T>(a, s); rs = b2_rsqrt<T>(s); }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ void b2_rho_rs<float>(float a, float s, float &q, float &rs) {
  rs = rsqrtf(s);
  q = a * (rs * rs);
}
#endif
