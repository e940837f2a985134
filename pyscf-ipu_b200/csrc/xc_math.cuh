// B3LYP per grid point: energy per particle and derivatives w.r.t. rho and sigma.
//
// Same functional as the reference's b3lyp (exchange_correlation/b3lyp.py:13-39):
//   0.08 Slater (lda.py:5, per particle) + 0.19 VWN (vwn.py:13-54, per volume)
//   + 0.72 B88 incl. its Slater part (b88.py:13-29) + 0.81 LYP (lyp.py:13-45),
// with rho clipped to [1e-9, 1e12], grad rho = 2 * rho[1:4] and sigma = |grad rho|^2 + 1e-20.
// The reference obtains vrho / vgamma with jax.value_and_grad; here the derivatives are
// written out analytically (derivation in the comments of each term).
#pragma once
#include "common.cuh"

template <typename T>
struct B2XcPoint { T exc, vrho, vgamma; };

// a / b: exact for float64; for float32 on the GPU the two-instruction approximate division
// (2 ulp; the functional's denominators stay far inside its range)
template <typename T> B2_HD T b2x_div(T a, T b) { return a / b; }
#ifdef __CUDA_ARCH__
template <> __device__ __forceinline__ float b2x_div<float>(float a, float b) { return __fdividef(a, b); }
#endif

// Exchange part (0.08 Slater + 0.72 B88) and correlation parts (0.19 VWN, 0.81 LYP);
// b2_b3lyp_point is their sum.  The split lets several threads share one grid point.
template <typename T>
B2_HD B2XcPoint<T> b2_b3lyp_x(T r0, T r1, T r2, T r3) {
  const T rho = r0 < (T)1e-9 ? (T)1e-9 : (r0 > (T)1e12 ? (T)1e12 : r0);
  const T gx = r1 + r1, gy = r2 + r2, gz = r3 + r3;
  const T sig = gx * gx + gy * gy + gz * gz + (T)1e-20;
  const T lr = log(rho);
  const T inv_rho = b2x_div<T>((T)1, rho);

  // --- Slater * 0.08: e = -exp(log(rho)/3 - 0.30305460484554375); d(rho e)/drho = 4/3 e
  const T e_lda = (T)-0.08 * exp(lr * (T)(1.0 / 3.0) - (T)0.30305460484554375);
  const T v_lda = (T)(4.0 / 3.0) * e_lda;

  // --- B88 * 0.72 (per volume, includes its Slater part): n = rho/2,
  //     x^2 = (sigma/4) n^{-8/3}, E = c3 n^{4/3} - 2 d n^{4/3} h(x), h = x^2 / Dn,
  //     Dn = 1 + 6 d x asinh(x), Dn' = 6 d (asinh x + x / sqrt(1+x^2))
  //     dE/drho = 1/2 [4/3 c3 n^{1/3} - 8/3 d n^{1/3} (h - x h')],
  //     h - x h' = x^2 (x Dn' - Dn) / Dn^2;  dE/dsigma = -(d/4) n^{-4/3} (h'/x),
  //     h'/x = (2 Dn - x Dn') / Dn^2
  const T d = (T)0.0042;
  const T c3 = (T)-1.8610514726982;                   // -(3/4) (6/pi)^{1/3} * 2
  const T n = rho * (T)0.5;
  const T ln = lr - (T)0.69314718055994531;
  const T n13 = exp(ln * (T)(1.0 / 3.0));
  const T n43 = n13 * n;
  const T x2 = sig * (T)0.25 * exp(ln * (T)(-8.0 / 3.0));
  const T x = sqrt(x2);
  const T ash = asinh(x);
  const T Dn = (T)1 + (T)6 * d * x * ash;
  const T Dnp = (T)6 * d * (ash + b2x_div<T>(x, sqrt((T)1 + x2)));
  const T h = b2x_div<T>(x2, Dn);
  const T E_b88 = c3 * n43 - (T)2 * d * n43 * h;
  const T hmxh = b2x_div<T>(x2 * (x * Dnp - Dn), Dn * Dn);
  const T hpx = b2x_div<T>((T)2 * Dn - x * Dnp, Dn * Dn);
  const T dEdn = (T)(4.0 / 3.0) * c3 * n13 - (T)(8.0 / 3.0) * d * n13 * hmxh;
  const T e_b88 = (T)0.72 * E_b88;
  const T v_b88 = (T)0.72 * (T)0.5 * dEdn;
  const T g_b88 = (T)0.72 * b2x_div<T>(-d * (T)0.25 * hpx, n43);

  B2XcPoint<T> o;
  o.exc = e_lda + e_b88 * inv_rho;
  o.vrho = v_lda + v_b88;
  o.vgamma = g_b88;
  return o;
}

template <typename T>
B2_HD B2XcPoint<T> b2_b3lyp_vwn(T r0, T r1, T r2, T r3) {
  const T rho = r0 < (T)1e-9 ? (T)1e-9 : (r0 > (T)1e12 ? (T)1e12 : r0);
  const T gx = r1 + r1, gy = r2 + r2, gz = r3 + r3;
  const T sig = gx * gx + gy * gy + gz * gz + (T)1e-20;
  const T lr = log(rho);
  const T rho13 = exp(lr * (T)(1.0 / 3.0));
  const T inv_rho = b2x_div<T>((T)1, rho);

  // --- VWN * 0.19: vwn(n) = n p1 G(s), s = (3/(4 pi n))^{1/6}
  //     G = log s + f [ log(s^2+p2 s+p3)/2 - (1/f+1) log(s-p0) ] + pre atan(c/(2s+p2))
  //     d vwn/dn = p1 [G - (s/6) G'(s)]
  const T p0 = (T)-0.10498, p1 = (T)0.0621813817393097900698817274255, p2 = (T)3.72744,
          p3 = (T)12.9352;
  const T f = (T)-1.0311676086789439;                // p0 p2 / (p0^2 + p0 p2 + p3) - 1
  const T c = (T)6.15199081975908;                    // sqrt(4 p3 - p2^2)
  const T pre = (T)0.6237121531215607;                 // p2 (1/c - p0 / ((p0^2+p0 p2+p3) c / (p2 + 2 p0)))
  const T log_s = -lr * (T)(1.0 / 6.0) + (T)-0.2387353263835302;    // log(3/(4pi))/6
  const T s = exp(log_s);
  const T X = s * s + p2 * s + p3;
  const T den = (T)2 * s + p2;
  const T z = b2x_div<T>(c, den);
  const T G = log_s + f * ((T)0.5 * log(X) - (T)(1.0 / -1.0311676086789439 + 1.0) * log(s - p0)) + pre * atan(z);
  const T Gp = b2x_div<T>((T)1, s) +
               f * (b2x_div<T>(den, (T)2 * X) - b2x_div<T>((T)(1.0 / -1.0311676086789439 + 1.0), s - p0)) +
               pre * b2x_div<T>(b2x_div<T>((T)-2 * c, den * den), (T)1 + z * z);
  const T e_vwn = (T)0.19 * rho * p1 * G;                      // per volume
  const T v_vwn = (T)0.19 * p1 * (G - s * (T)(1.0 / 6.0) * Gp);

  B2XcPoint<T> o;
  o.exc = e_vwn * inv_rho;
  o.vrho = v_vwn;
  o.vgamma = (T)0;
  return o;
}

template <typename T>
B2_HD B2XcPoint<T> b2_b3lyp_lyp(T r0, T r1, T r2, T r3) {
  const T rho = r0 < (T)1e-9 ? (T)1e-9 : (r0 > (T)1e12 ? (T)1e12 : r0);
  const T gx = r1 + r1, gy = r2 + r2, gz = r3 + r3;
  const T sig = gx * gx + gy * gy + gz * gz + (T)1e-20;
  const T lr = log(rho);
  const T rho13 = exp(lr * (T)(1.0 / 3.0));
  const T inv_rho = b2x_div<T>((T)1, rho);

  // --- LYP * 0.81: t = n^{-1/3}, P = 1/(1 + D t), w = exp(-C t) P, dl = t (C + D P)
  //     R = -A n P - A B CF w n + (A B / 72) w sigma n^{-5/3} (3 + 7 dl)
  //     P' = D P^2 t/(3n), w' = w dl/(3n), dl' = (D^2 P^2 t^2 - dl)/(3n)
  const T A = (T)0.04918, B = (T)0.132, C = (T)0.2533, D = (T)0.349;
  const T CF = (T)2.8712340001881918;                 // 0.3 (3 pi^2)^{2/3}
  const T t = b2x_div<T>((T)1, rho13);
  const T P = b2x_div<T>((T)1, (T)1 + D * t);
  const T w = exp(-C * t) * P;
  const T dl = t * (C + D * P);
  const T n53 = t * t * t * t * t;                     // rho^{-5/3}
  const T q = (T)3 + (T)7 * dl;
  const T R = -A * rho * P - A * B * CF * w * rho + (T)(0.04918 * 0.132 / 72.0) * w * sig * n53 * q;
  const T i3n = inv_rho * (T)(1.0 / 3.0);
  const T Pp = D * P * P * t * i3n;
  const T wp = w * dl * i3n;
  const T dlp = (D * D * P * P * t * t - dl) * i3n;
  const T dRdn = -A * (P + rho * Pp) - A * B * CF * (w + rho * wp) +
                 (T)(0.04918 * 0.132 / 72.0) * sig *
                     (wp * n53 * q - (T)(5.0 / 3.0) * w * n53 * inv_rho * q + (T)7 * w * n53 * dlp);
  const T dRdg = (T)(0.04918 * 0.132 / 72.0) * w * n53 * q;
  const T e_lyp = (T)0.81 * R;
  const T v_lyp = (T)0.81 * dRdn;
  const T g_lyp = (T)0.81 * dRdg;

  B2XcPoint<T> o;
  o.exc = e_lyp * inv_rho;
  o.vrho = v_lyp;
  o.vgamma = g_lyp;
  return o;
}

template <typename T>
B2_HD B2XcPoint<T> b2_b3lyp_c(T r0, T r1, T r2, T r3) {
  const B2XcPoint<T> a = b2_b3lyp_vwn<T>(r0, r1, r2, r3), b = b2_b3lyp_lyp<T>(r0, r1, r2, r3);
  B2XcPoint<T> o;
  o.exc = a.exc + b.exc;
  o.vrho = a.vrho + b.vrho;
  o.vgamma = a.vgamma + b.vgamma;
  return o;
}

template <typename T>
B2_HD B2XcPoint<T> b2_b3lyp_point(T r0, T r1, T r2, T r3) {
  const B2XcPoint<T> x = b2_b3lyp_x<T>(r0, r1, r2, r3), c = b2_b3lyp_c<T>(r0, r1, r2, r3);
  B2XcPoint<T> o;
  o.exc = x.exc + c.exc;
  o.vrho = x.vrho + c.vrho;
  o.vgamma = x.vgamma + c.vgamma;
  return o;
}
