// Two-electron integrals (ij|kl) for s/p Gaussians.
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
// every bra/ket combination (the f[n] and g terms below).  The reference computes the same
// integrals by Rys quadrature (int2e_sph.cpp:1785-1892, 2452-2719); results agree to
// rounding.
//
// Shell-quartet evaluation: one thread computes every component (i j | k l) of one bra shell
// pair IJ against one ket shell pair KL of a fixed angular class; the primitive-quartet
// quantities (Boys values, X = P - Q, prefactor) are computed once per primitive quartet and
// shared by all components.
#pragma once
#include "boys.cuh"
#include "plan_host.hpp"

// CI < 0: all bra i components in this thread; CI >= 0: only component CI (float64 form
// splits p bras over 3 threads to bound register use).
template <typename T, int LI, int LJ, int LK, int LL, int CI>
struct B2Sq {
  static constexpr int NI = LI ? (CI < 0 ? 3 : 1) : 1;
  static constexpr int NJ = LJ ? 3 : 1, NK = LK ? 3 : 1, NL = LL ? 3 : 1;
  static constexpr int L = LI + LJ + LK + LL;

  B2_HD static void zero(T acc[NI][NJ][NK][NL]) {
#pragma unroll
    for (int a = 0; a < NI; ++a)
#pragma unroll
      for (int b = 0; b < NJ; ++b)
#pragma unroll
        for (int c = 0; c < NK; ++c)
#pragma unroll
          for (int d = 0; d < NL; ++d) acc[a][b][c][d] = (T)0;
  }

  // one primitive quartet (bra primitive pair Bp, ket primitive pair Q) added to acc
  B2_HD static void quartet(const B2PairPrim<T> &Bp, const B2PairPrim<T> &Q, const T *__restrict__ btab,
                            T acc[NI][NJ][NK][NL]) {
    const T eta = Q.zeta;
    const T v = Q.h2z;
    const T QC[3] = {Q.PAx, Q.PAy, Q.PAz};
    const T QD[3] = {Q.PBx, Q.PBy, Q.PBz};

    const T zeta = Bp.zeta;
    const T u = Bp.h2z;
    const T sig = zeta + eta;
    T rho, rs;                                // rho = zeta eta / sig, rs = 1 / sqrt(sig)
    b2_rho_rs<T>(zeta * eta, sig, rho, rs);
    const T X[3] = {Bp.Px - Q.Px, Bp.Py - Q.Py, Bp.Pz - Q.Pz};
    const T tt = rho * (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    const T pref = Bp.K * Q.K * rs;
    T F[L + 1];
    b2_boys<T, L, T>(tt, btab, F);
    T f[L + 3];
    {
      T m2r = (T)-2 * rho, s = pref;
#pragma unroll
      for (int n = 0; n <= L; ++n) { f[n] = s * F[n]; s *= m2r; }
      f[L + 1] = (T)0;
      f[L + 2] = (T)0;
    }
    const T PA[3] = {Bp.PAx, Bp.PAy, Bp.PAz};
    const T PB[3] = {Bp.PBx, Bp.PBy, Bp.PBz};
#pragma unroll
    for (int ia = 0; ia < NI; ++ia) {
      const int a = CI < 0 ? ia : CI;
      const T sa = LI ? PA[a] : (T)1;
      const T xa = LI ? X[a] : (T)0;
#pragma unroll
      for (int b = 0; b < NJ; ++b) {
        const T sb = LJ ? PB[b] : (T)1;
        const T xb = LJ ? X[b] : (T)0;
        const T abf = (LI && LJ && a == b) ? (T)1 : (T)0;
        const T E0 = sa * sb + abf * u;
        const T Ea = LI ? sb * u : (T)0;
        const T Eb = LJ ? sa * u : (T)0;
        const T Eab = (LI && LJ) ? u * u : (T)0;
        const T lin = Ea * xa + Eb * xb + Eab * abf;
        const T quad = Eab * xa * xb;
        const T g0 = E0 * f[0] + lin * f[1] + quad * f[2];
        if (LK == 0 && LL == 0) {
          acc[ia][b][0][0] += g0;
          continue;
        }
        const T g1 = E0 * f[1] + lin * f[2] + quad * f[3];
        const T A1 = Ea * f[1] + Eab * xb * f[2];
        const T B1 = Eb * f[1] + Eab * xa * f[2];
        T Bc[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          Bc[c] = X[c] * g1 + ((LI && c == a) ? A1 : (T)0) + ((LJ && c == b) ? B1 : (T)0);
        if (LK && !LL) {
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[ia][b][c][0] += QC[c] * g0 - v * Bc[c];
        } else if (!LK && LL) {
#pragma unroll
          for (int d = 0; d < 3; ++d) acc[ia][b][0][d] += QD[d] * g0 - v * Bc[d];
        } else {
          const T g2 = E0 * f[2] + lin * f[3] + quad * f[4];
          const T A2 = Ea * f[2] + Eab * xb * f[3];
          const T B2 = Eb * f[2] + Eab * xa * f[3];
          const T W = Eab * f[2];
          T V2[3];
#pragma unroll
          for (int c = 0; c < 3; ++c)
            V2[c] = ((LI && c == a) ? A2 : (T)0) + ((LJ && c == b) ? B2 : (T)0);
          const T vv = v * v;
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const int wcd = (LI && LJ) ? ((c == a && d == b) ? 1 : 0) + ((d == a && c == b) ? 1 : 0) : 0;
              const T Bcd = (c == d ? g1 : (T)0) + X[c] * X[d] * g2 + X[d] * V2[c] + X[c] * V2[d] +
                            (wcd ? W * (T)wcd : (T)0);
              const T F0 = QC[c] * QD[d] + (c == d ? v : (T)0);
              acc[ia][b][c][d] += F0 * g0 - v * (QD[d] * Bc[c] + QC[c] * Bc[d]) + vv * Bcd;
            }
        }
      }
    }
  }

  B2_HD static void eval(const B2PairPrim<T> *__restrict__ bra, int nb,
                         const B2PairPrim<T> *__restrict__ ket, const T *__restrict__ btab,
                         T acc[NI][NJ][NK][NL]) {
    zero(acc);
    for (int q = 0; q < B2_MAXPP; ++q) {
      const B2PairPrim<T> Q = ket[q];
      if (Q.K == (T)0) break;                 // packed: the rest of the pair is inert
      for (int p = 0; p < nb; ++p) quartet(bra[p], Q, btab, acc);
    }
  }

  // write the block into one molecule's s8 list (only entries whose row ij belongs to this bra)
  template <typename TO>
  B2_HD static void store(TO *out, const B2PairInfo &bp, const B2PairInfo &kp,
                          const T acc[NI][NJ][NK][NL]) {
#pragma unroll
    for (int ia = 0; ia < NI; ++ia) {
      const int i = bp.ao0I + (CI < 0 ? ia : CI);
#pragma unroll
      for (int b = 0; b < NJ; ++b) {
        const int j = bp.ao0J + b;
        if (bp.I == bp.J && j > i) continue;
        const long long ij = b2_tri(i) + j;
        const long long rowbase = b2_tri(ij);
#pragma unroll
        for (int c = 0; c < NK; ++c) {
          const int k = kp.ao0I + c;
#pragma unroll
          for (int d = 0; d < NL; ++d) {
            const int l = kp.ao0J + d;
            if (kp.I == kp.J && l > k) continue;
            const long long kl = b2_tri(k) + l;
            if (kl > ij) continue;
            out[rowbase + kl] = (TO)acc[ia][b][c][d];
          }
        }
      }
    }
  }

  template <typename TO>
  B2_HD static void run(const B2PairPrim<T> *bra, int nb, const B2PairPrim<T> *ket,
                        const T *btab, TO *out, const B2PairInfo &bp, const B2PairInfo &kp) {
    T acc[NI][NJ][NK][NL];
    eval(bra, nb, ket, btab, acc);
    store<TO>(out, bp, kp, acc);
  }
};

// work item of the ERI kernel: one warp = one bra shell pair x a chunk of kets of one class
struct B2EriTask {
  int mol, IJ, cls, start, count, sub;
};

// task list (host): bra shell pairs x ket classes, kets split into chunks of `chunk`;
// split_p: split p-shell bras I by component (float64 form)
// grouped by class combination g = bra class * 4 + ket class; goff (17 entries) = group starts
static void b2_eri_tasks(const B2PlanHost &P, int chunk, bool split_p, std::vector<B2EriTask> &out,
                         std::vector<long long> *goff = nullptr) {
  // two passes over (molecule, bra pair, ket class): count tasks per group, then place them
  std::vector<long long> g(17, 0);
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<long long> pos(g.begin(), g.end() - 1);
    for (int m = 0; m < P.nmol; ++m) {
      const B2MolDev &md = P.mols[m];
      for (int IJ = 0; IJ < md.nsp; ++IJ) {
        const B2PairInfo &pi = P.pinfo[md.sp_off + IJ];
        const int spcut = (int)b2_tri(pi.I) + pi.I;
        const int nsub = (split_p && pi.lI) ? 3 : 1;
        for (int c = 0; c < 4; ++c) {
          const int cnt = P.cls_cnt[4ll * md.sp_off + (long long)c * md.nsp + spcut];
          const int grp = (pi.lI + 2 * pi.lJ) * 4 + c;
          if (pass == 0) {
            g[grp + 1] += (long long)((cnt + chunk - 1) / chunk) * nsub;
            continue;
          }
          for (int s0 = 0; s0 < cnt; s0 += chunk)
            for (int sub = 0; sub < nsub; ++sub)
              out[pos[grp]++] = B2EriTask{m, IJ, c, s0, std::min(chunk, cnt - s0), nsub > 1 ? sub : -1};
        }
      }
    }
    if (pass == 0) {
      for (int k = 0; k < 16; ++k) g[k + 1] += g[k];
      out.assign((size_t)g[16], B2EriTask{});
    }
  }
  if (goff) *goff = g;
}

// dispatch on (bra class, ket class, sub) to the specialised evaluator
template <typename T, int LI, int LJ, int LK, int LL, typename TO>
B2_HD void b2_sq_sub(int sub, const B2PairPrim<T> *bra, int nb, const B2PairPrim<T> *ket,
                     const T *btab, TO *out, const B2PairInfo &bp, const B2PairInfo &kp) {
  if (LI && sub >= 0) {
    switch (sub) {
      case 0: B2Sq<T, LI, LJ, LK, LL, 0>::template run<TO>(bra, nb, ket, btab, out, bp, kp); break;
      case 1: B2Sq<T, LI, LJ, LK, LL, 1>::template run<TO>(bra, nb, ket, btab, out, bp, kp); break;
      default: B2Sq<T, LI, LJ, LK, LL, 2>::template run<TO>(bra, nb, ket, btab, out, bp, kp); break;
    }
  } else {
    B2Sq<T, LI, LJ, LK, LL, -1>::template run<TO>(bra, nb, ket, btab, out, bp, kp);
  }
}

template <typename T, int LI, int LJ, typename TO>
B2_HD void b2_sq_ket(int cls, int sub, const B2PairPrim<T> *bra, int nb, const B2PairPrim<T> *ket,
                     const T *btab, TO *out, const B2PairInfo &bp, const B2PairInfo &kp) {
  switch (cls) {
    case 0: b2_sq_sub<T, LI, LJ, 0, 0, TO>(sub, bra, nb, ket, btab, out, bp, kp); break;
    case 1: b2_sq_sub<T, LI, LJ, 1, 0, TO>(sub, bra, nb, ket, btab, out, bp, kp); break;
    case 2: b2_sq_sub<T, LI, LJ, 0, 1, TO>(sub, bra, nb, ket, btab, out, bp, kp); break;
    default: b2_sq_sub<T, LI, LJ, 1, 1, TO>(sub, bra, nb, ket, btab, out, bp, kp); break;
  }
}

template <typename T, typename TO>
B2_HD void b2_sq_dispatch(int bcls, int cls, int sub, const B2PairPrim<T> *bra, int nb,
                          const B2PairPrim<T> *ket, const T *btab, TO *out,
                          const B2PairInfo &bp, const B2PairInfo &kp) {
  switch (bcls) {
    case 0: b2_sq_ket<T, 0, 0, TO>(cls, sub, bra, nb, ket, btab, out, bp, kp); break;
    case 1: b2_sq_ket<T, 1, 0, TO>(cls, sub, bra, nb, ket, btab, out, bp, kp); break;
    case 2: b2_sq_ket<T, 0, 1, TO>(cls, sub, bra, nb, ket, btab, out, bp, kp); break;
    default: b2_sq_ket<T, 1, 1, TO>(cls, sub, bra, nb, ket, btab, out, bp, kp); break;
  }
}
