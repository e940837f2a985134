// Two-electron integrals (ij|kl) for s/p Gaussians, one bra AO pair against all
// components of one ket shell pair.
//
// Formulation (this project's own, from the McMurchie-Davidson Hermite expansion):
// every s/p bra factor (r-A)_a = (r-P)_a + PA_a, and (r-P)_a exp(-zeta|r-P|^2) =
// (1/2zeta) d/dP_a exp(...), so a primitive bra pair is a short polynomial in
// derivatives with respect to P:
//   E0 + Ea d_alpha + Eb d_beta + Eab d_alpha d_beta
//   (E0 = sa sb + [a.b] u, Ea = sb u, Eb = sa u, Eab = u^2, u = 1/(2 zeta),
//    sa = PA.alpha or 1 for s, sb = PB.beta or 1 for s);
// the ket likewise with u -> v = 1/(2 eta), derivatives taken w.r.t. Q = -X.
// Derivatives of the base integral f_0(X) = pref F_0(rho |X|^2) follow from
// d_c f_n = X_c f_{n+1}, f_n = pref (-2 rho)^n F_n(rho X^2), which gives closed forms for
// every bra/ket combination (``g_n``, ``V_n`` below).  The reference computes the same
// integrals by Rys quadrature (int2e_sph.cpp:1785-1892, 2452-2719); results agree to
// rounding.
#pragma once
#include "boys.cuh"

// bra primitive data with the row's bra components folded in (per CTA)
template <typename T>
struct B2BraPrim {
  T zeta, Px, Py, Pz, K, E0, Ea, Eb, Eab, xsel;   // xsel: padding to 80 bytes (float64)
};

template <typename T>
B2_HD T b2_sel3(int c, T x, T y, T z) { return c == 0 ? x : (c == 1 ? y : z); }

template <typename T, int LI, int LJ>
B2_HD void b2_make_bra(const B2PairPrim<T> &P, int ci, int cj, B2BraPrim<T> &B) {
  T u = (T)0.5 / P.zeta;
  T sa = LI ? b2_sel3<T>(ci, P.PAx, P.PAy, P.PAz) : (T)1;
  T sb = LJ ? b2_sel3<T>(cj, P.PBx, P.PBy, P.PBz) : (T)1;
  T ab = (LI && LJ && ci == cj) ? (T)1 : (T)0;
  B.zeta = P.zeta; B.Px = P.Px; B.Py = P.Py; B.Pz = P.Pz; B.K = P.K;
  B.E0 = sa * sb + ab * u;
  B.Ea = LI ? sb * u : (T)0;
  B.Eb = LJ ? sa * u : (T)0;
  B.Eab = (LI && LJ) ? u * u : (T)0;
  B.xsel = 0;
}

// acc[ck][cl] += (i j | k l) for all ket components of one ket shell pair.
// bra: nb primitive pairs (already folded), ket: nk primitive pairs of the ket shell pair.
template <typename T, int LI, int LJ, int LK, int LL>
B2_HD void b2_eri_item(const B2BraPrim<T> *__restrict__ bra, int nb,
                       const B2PairPrim<T> *__restrict__ ket, int nk, int ci, int cj,
                       const double *__restrict__ btab, T acc[3][3]) {
  constexpr int L = LI + LJ + LK + LL;
  const T abf = (LI && LJ && ci == cj) ? (T)1 : (T)0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) acc[a][b] = (T)0;
  for (int q = 0; q < nk; ++q) {
    const B2PairPrim<T> Q = ket[q];
    if (Q.K == (T)0) continue;
    const T eta = Q.zeta;
    const T v = (T)0.5 / eta;
    const T QC[3] = {Q.PAx, Q.PAy, Q.PAz};
    const T QD[3] = {Q.PBx, Q.PBy, Q.PBz};
    for (int p = 0; p < nb; ++p) {
      const B2BraPrim<T> &B = bra[p];
      const T zeta = B.zeta;
      const T sig = zeta + eta;
      const T rho = zeta * eta / sig;
      const T X[3] = {B.Px - Q.Px, B.Py - Q.Py, B.Pz - Q.Pz};
      const T tt = rho * (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
      const T pref = B.K * Q.K / sqrt(sig);
      T F[L + 1];
      b2_boys<T, L>(tt, btab, F);
      T f[L + 3];
      T m2r = (T)-2 * rho, s = pref;
#pragma unroll
      for (int n = 0; n <= L; ++n) { f[n] = s * F[n]; s *= m2r; }
      f[L + 1] = (T)0;
      f[L + 2] = (T)0;
      const T xa = LI ? b2_sel3<T>(ci, X[0], X[1], X[2]) : (T)0;
      const T xb = LJ ? b2_sel3<T>(cj, X[0], X[1], X[2]) : (T)0;
      const T lin = B.Ea * xa + B.Eb * xb + B.Eab * abf;
      const T quad = B.Eab * xa * xb;
      const T g0 = B.E0 * f[0] + lin * f[1] + quad * f[2];
      if (LK == 0 && LL == 0) {
        acc[0][0] += g0;
        continue;
      }
      const T g1 = B.E0 * f[1] + lin * f[2] + quad * f[3];
      const T A1 = B.Ea * f[1] + B.Eab * xb * f[2];
      const T B1 = B.Eb * f[1] + B.Eab * xa * f[2];
      T Bc[3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        Bc[c] = X[c] * g1 + ((LI && c == ci) ? A1 : (T)0) + ((LJ && c == cj) ? B1 : (T)0);
      if (LK && !LL) {
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c][0] += QC[c] * g0 - v * Bc[c];
      } else if (!LK && LL) {
#pragma unroll
        for (int d = 0; d < 3; ++d) acc[0][d] += QD[d] * g0 - v * Bc[d];
      } else {
        const T g2 = B.E0 * f[2] + lin * f[3] + quad * f[4];
        const T A2 = B.Ea * f[2] + B.Eab * xb * f[3];
        const T B2 = B.Eb * f[2] + B.Eab * xa * f[3];
        const T W = B.Eab * f[2];
        T V2[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          V2[c] = ((LI && c == ci) ? A2 : (T)0) + ((LJ && c == cj) ? B2 : (T)0);
        const T vv = v * v;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            T wcd = (LI && LJ) ? (T)((c == ci && d == cj) ? 1 : 0) + (T)((d == ci && c == cj) ? 1 : 0)
                               : (T)0;
            T Bcd = (c == d ? g1 : (T)0) + X[c] * X[d] * g2 + X[d] * V2[c] + X[c] * V2[d] + W * wcd;
            T F0 = QC[c] * QD[d] + (c == d ? v : (T)0);
            acc[c][d] += F0 * g0 - v * (QD[d] * Bc[c] + QC[c] * Bc[d]) + vv * Bcd;
          }
      }
    }
  }
}
