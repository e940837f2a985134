// Two-electron part of the RKS nuclear gradient for s / p shells (host and device code).
//
// The reference's gradient (nanoDFT.py:403-426) contracts int2e_ip1 = (d/dA_x i j|k l) with the
// density: vj = -sum (d_i j|k l) D_lk, vk = -sum (d_i j|k l) D_jk, de_A += 2 <vj - hyb/2 vk,
// D>_{i on A}.  Over all ordered index quartets that is
//
//   dE_2e / dR = sum_{ijkl} d(ij|kl)/dR  Gamma_ijkl,   Gamma = 1/2 D_ij D_kl - hyb/4 D_il D_jk,
//
// the derivative at fixed D of E_2e = 1/2 <D, J> - hyb/4 <D, K>.  For one shell quartet
// (I J | K L) this file evaluates the derivatives with respect to the centres of I, J and K and
// takes the fourth from translation invariance (the four sum to zero).  A primitive's
// derivative is d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}; the integrals over Cartesian
// Gaussians come from the Obara-Saika vertical recursion (Obara & Saika, J. Chem. Phys. 84,
// 3963 (1986)) for [e 0 | f 0], contracted with weights 1, 2 alpha, 2 beta, 2 gamma, then the
// Head-Gordon-Pople horizontal recursion (J. Chem. Phys. 89, 5777 (1988)) moves angular
// momentum to the second centre of each pair.  Shells are s or p (l <= 1), so Cartesian
// components up to l = 3 occur.
#pragma once
#include "common.cuh"
#include "boys.cuh"
#include "plan_host.hpp"
#include "xc_math.cuh"

#define B2G_NC 20                  // Cartesian components of l = 0..3
#define B2G_MMAX 6                 // Boys orders 0..5

B2_HD constexpr int b2g_cstart(int l) { return l * (l + 1) * (l + 2) / 6; }
B2_HD constexpr int b2g_ncart(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }   // components of 0..l
// index of the Cartesian (x, y, z) among all components of l = 0..3 (order within a shell:
// x descending, then y descending)
B2_HD constexpr int b2g_cidx(int x, int y, int z) {
  const int l = x + y + z;
  return b2g_cstart(l) + (l - x) * (l - x + 1) / 2 + z;
}
B2_HD constexpr void b2g_cart(int idx, int &x, int &y, int &z) {
  int l = 0;
  while (b2g_cstart(l + 1) <= idx) ++l;
  int r = idx - b2g_cstart(l);
  int lx = l;                                    // r = (l - x)(l - x + 1)/2 + z
  while (true) {
    const int k = l - lx, base = k * (k + 1) / 2;
    if (r < base + k + 1) { z = r - base; x = lx; y = l - x - z; return; }
    --lx;
  }
}

B2_HD double b2g_binom(int n, int k) { return (n == 2 && k == 1) ? 2.0 : 1.0; }   // n <= 2 here
template <typename T> B2_HD T b2g_pow(T x, int n) { T r = (T)1; for (int i = 0; i < n; ++i) r *= x; return r; }

// Boys F_0..F_L (L <= 5) from the float64 table (same scheme as b2_boys)
template <typename T>
B2_HD void b2g_boys(int L, T t, const T *btab, T *F) {
  switch (L) {
    case 0: b2_boys<T, 0, T>(t, btab, F); break;
    case 1: b2_boys<T, 1, T>(t, btab, F); break;
    case 2: b2_boys<T, 2, T>(t, btab, F); break;
    case 3: b2_boys<T, 3, T>(t, btab, F); break;
    case 4: b2_boys<T, 4, T>(t, btab, F); break;
    default: b2_boys<T, 5, T>(t, btab, F); break;
  }
}

// contracted [e 0 | f 0] for e over l <= LE, f over l <= LF, with the weightings of the bra
// pass (KET false; w = 0: plain, 1: x 2 alpha of the first bra primitive, 2: x 2 beta of the
// second) or of the ket pass (KET true; w = 0: plain, 1: x 2 gamma of the first ket
// primitive).  Shells a, b, c, d (their coefficients include the angular factors).  The
// array sizes follow the class, so a GPU thread holds no more than the class needs.
template <typename T, int LE, int LF, bool KET>
B2_HD void b2g_e0f0(const B2Shell &a, const B2Shell &b, const B2Shell &c, const B2Shell &d,
                    const T *btab, T (*acc)[b2g_ncart(LE)][b2g_ncart(LF)]) {
  constexpr int ne = b2g_ncart(LE), nf = b2g_ncart(LF), L = LE + LF, NW = KET ? 2 : 3;
  const int le = LE, lf = LF;
  for (int w = 0; w < NW; ++w)
    for (int i = 0; i < ne; ++i)
      for (int j = 0; j < nf; ++j) acc[w][i][j] = (T)0;
  T AB2 = 0, CD2 = 0;
  for (int x = 0; x < 3; ++x) {
    AB2 += (T)((a.R[x] - b.R[x]) * (a.R[x] - b.R[x]));
    CD2 += (T)((c.R[x] - d.R[x]) * (c.R[x] - d.R[x]));
  }
  for (int pa = 0; pa < a.nprim; ++pa)
    for (int pb = 0; pb < b.nprim; ++pb) {
      const T al = (T)a.exp[pa], be = (T)b.exp[pb], z = al + be;
      T P[3], PA[3];
      for (int x = 0; x < 3; ++x) {
        P[x] = (al * (T)a.R[x] + be * (T)b.R[x]) / z;
        PA[x] = P[x] - (T)a.R[x];
      }
      const T Kab = exp(-al * be / z * AB2) * (T)a.coef[pa] * (T)b.coef[pb];
      for (int pc = 0; pc < c.nprim; ++pc)
        for (int pd = 0; pd < d.nprim; ++pd) {
          const T ga = (T)c.exp[pc], de = (T)d.exp[pd], e = ga + de;
          T Q[3], QC[3], WP[3], WQ[3], PQ2 = 0;
          for (int x = 0; x < 3; ++x) {
            Q[x] = (ga * (T)c.R[x] + de * (T)d.R[x]) / e;
            QC[x] = Q[x] - (T)c.R[x];
            const T W = (z * P[x] + e * Q[x]) / (z + e);
            WP[x] = W - P[x];
            WQ[x] = W - Q[x];
            PQ2 += (P[x] - Q[x]) * (P[x] - Q[x]);
          }
          const T rho = z * e / (z + e);
          const T Kcd = exp(-ga * de / e * CD2) * (T)c.coef[pc] * (T)d.coef[pd];
          // 2 pi^(5/2) / (z e sqrt(z + e))
          const T pref = (T)34.98683665524972 / (z * e * sqrt(z + e)) * Kab * Kcd;
          T F[B2G_MMAX];
          b2g_boys<T>(L, rho * PQ2, btab, F);
          T v[ne][nf][L + 1];
          for (int m = 0; m <= L; ++m) v[0][0][m] = pref * F[m];
          for (int l1 = 1; l1 <= le; ++l1)                // bra vertical recursion
            for (int ie = b2g_cstart(l1); ie < b2g_cstart(l1 + 1); ++ie) {
              int ex, ey, ez;
              b2g_cart(ie, ex, ey, ez);
              const int dd = ex ? 0 : (ey ? 1 : 2);
              int e1[3] = {ex, ey, ez};
              e1[dd]--;
              const int i1 = b2g_cidx(e1[0], e1[1], e1[2]);
              int i2 = -1;
              if (e1[dd] > 0) {
                int e2[3] = {e1[0], e1[1], e1[2]};
                e2[dd]--;
                i2 = b2g_cidx(e2[0], e2[1], e2[2]);
              }
              for (int m = 0; m <= L - l1; ++m) {
                T t = PA[dd] * v[i1][0][m] + WP[dd] * v[i1][0][m + 1];
                if (i2 >= 0) t += (T)e1[dd] / (2 * z) * (v[i2][0][m] - rho / z * v[i2][0][m + 1]);
                v[ie][0][m] = t;
              }
            }
          for (int l2 = 1; l2 <= lf; ++l2)                // ket vertical recursion
            for (int jf = b2g_cstart(l2); jf < b2g_cstart(l2 + 1); ++jf) {
              int fx, fy, fz;
              b2g_cart(jf, fx, fy, fz);
              const int dd = fx ? 0 : (fy ? 1 : 2);
              int f1[3] = {fx, fy, fz};
              f1[dd]--;
              const int j1 = b2g_cidx(f1[0], f1[1], f1[2]);
              int j2 = -1;
              if (f1[dd] > 0) {
                int f2[3] = {f1[0], f1[1], f1[2]};
                f2[dd]--;
                j2 = b2g_cidx(f2[0], f2[1], f2[2]);
              }
              for (int ie = 0; ie < ne; ++ie) {
                int ex, ey, ez;
                b2g_cart(ie, ex, ey, ez);
                const int ec[3] = {ex, ey, ez};
                const int l1 = ex + ey + ez;
                int i3 = -1;
                if (ec[dd] > 0) {
                  int e3[3] = {ex, ey, ez};
                  e3[dd]--;
                  i3 = b2g_cidx(e3[0], e3[1], e3[2]);
                }
                for (int m = 0; m <= L - l1 - l2; ++m) {
                  T t = QC[dd] * v[ie][j1][m] + WQ[dd] * v[ie][j1][m + 1];
                  if (j2 >= 0) t += (T)f1[dd] / (2 * e) * (v[ie][j2][m] - rho / e * v[ie][j2][m + 1]);
                  if (i3 >= 0) t += (T)ec[dd] / (2 * (z + e)) * v[i3][j1][m + 1];
                  v[ie][jf][m] = t;
                }
              }
            }
          const T wt[3] = {(T)1, KET ? 2 * ga : 2 * al, 2 * be};
          for (int w = 0; w < NW; ++w)
            for (int i = 0; i < ne; ++i)
              for (int j = 0; j < nf; ++j) acc[w][i][j] += wt[w] * v[i][j][0];
        }
    }
}

// The GPU kernels' form of the vertical recursion (csrc/grad.cu): the steps of b2g_e0f0 for one
// class, tabulated (target, sources, direction, integer factors, last m) so that lanes can share
// a level's steps; the host-check build runs the same table in order against b2g_e0f0.
struct B2gOp {                      // one recursion step: v[dst + m] from v[s1..], v[s2..], v[s3..]
  short dst, s1, s2, s3;            // flat offsets (s2 / s3 < 0: term absent)
  signed char dd, c1, c3, mmax;     // direction, integer factors of the s2 / s3 terms, last m
};
template <int LE, int LF, int L>
struct B2gVrr {                     // the recursion for [e0|f0]^(m), e up to LE, f up to LF
  static constexpr int NE = b2g_ncart(LE), NF = b2g_ncart(LF), SM = L + 1, SE = NF * SM;
  static constexpr int NV = NE * SE;                        // doubles of v[e][f][m]
  static constexpr int NOB = NE - 1;                        // bra steps: e = 1..NE-1, f = 0
  static constexpr int NOK = (NF - 1) * NE;                 // ket steps: f = 1..NF-1, every e
  static constexpr int NOP = NOB + NOK;
  static constexpr int NACC = NE * NF;                      // (e, f) entries of the result
  // step o of the table (bra steps by e, then ket steps by f with e inner: levels in order)
  B2_HD static constexpr B2gOp op(int o) {
    B2gOp r{};
    r.s3 = -1;
    r.c3 = 0;
    if (o < NOB) {
      const int ie = o + 1;
      int ex = 0, ey = 0, ez = 0;
      b2g_cart(ie, ex, ey, ez);
      const int e[3] = {ex, ey, ez};
      const int dd = ex ? 0 : (ey ? 1 : 2);
      int e1[3] = {e[0], e[1], e[2]};
      e1[dd]--;
      r.dst = (short)(ie * SE);
      r.s1 = (short)(b2g_cidx(e1[0], e1[1], e1[2]) * SE);
      r.s2 = -1;
      r.c1 = (signed char)e1[dd];
      if (e1[dd] > 0) {
        int e2[3] = {e1[0], e1[1], e1[2]};
        e2[dd]--;
        r.s2 = (short)(b2g_cidx(e2[0], e2[1], e2[2]) * SE);
      }
      r.dd = (signed char)dd;
      r.mmax = (signed char)(L - (ex + ey + ez));
    } else {
      const int q = o - NOB, jf = 1 + q / NE, ie = q - (q / NE) * NE;
      int fx = 0, fy = 0, fz = 0, ex = 0, ey = 0, ez = 0;
      b2g_cart(jf, fx, fy, fz);
      b2g_cart(ie, ex, ey, ez);
      const int dd = fx ? 0 : (fy ? 1 : 2);
      int f1[3] = {fx, fy, fz};
      f1[dd]--;
      const int j1 = b2g_cidx(f1[0], f1[1], f1[2]);
      const int ec[3] = {ex, ey, ez};
      r.dst = (short)(ie * SE + jf * SM);
      r.s1 = (short)(ie * SE + j1 * SM);
      r.s2 = -1;
      r.c1 = (signed char)f1[dd];
      if (f1[dd] > 0) {
        int f2[3] = {f1[0], f1[1], f1[2]};
        f2[dd]--;
        r.s2 = (short)(ie * SE + b2g_cidx(f2[0], f2[1], f2[2]) * SM);
      }
      if (ec[dd] > 0) {
        int e3[3] = {ex, ey, ez};
        e3[dd]--;
        r.s3 = (short)(b2g_cidx(e3[0], e3[1], e3[2]) * SE + j1 * SM);
        r.c3 = (signed char)ec[dd];
      }
      r.dd = (signed char)dd;
      r.mmax = (signed char)(L - (ex + ey + ez) - (fx + fy + fz));   // < 0: nothing to do
    }
    return r;
  }
};

// (a b | c d) over Cartesian exponent triplets (a, b on the bra centres A, B; c, d on C, D) from
// contracted [e 0 | f 0] (weighting w): horizontal recursion (a b+1_x| = (a+1_x b| + AB_x (a b|
template <typename T, int NE, int NF>
B2_HD T b2g_hrr(const T (*acc)[NE][NF], int w, const int *ea, const int *eb, const int *ec, const int *ed,
                const T *AB, const T *CD) {
  // expand b onto a: sum over binomial terms of (a + b')|, with weight AB^(b - b')
  T s = 0;
  for (int bx = 0; bx <= eb[0]; ++bx)
    for (int by = 0; by <= eb[1]; ++by)
      for (int bz = 0; bz <= eb[2]; ++bz) {
        const T cb = (T)b2g_binom(eb[0], bx) * b2g_binom(eb[1], by) * b2g_binom(eb[2], bz) *
                     b2g_pow(AB[0], eb[0] - bx) * b2g_pow(AB[1], eb[1] - by) * b2g_pow(AB[2], eb[2] - bz);
        const int ie = b2g_cidx(ea[0] + bx, ea[1] + by, ea[2] + bz);
        for (int dx = 0; dx <= ed[0]; ++dx)
          for (int dy = 0; dy <= ed[1]; ++dy)
            for (int dz = 0; dz <= ed[2]; ++dz) {
              const T cd = (T)b2g_binom(ed[0], dx) * b2g_binom(ed[1], dy) * b2g_binom(ed[2], dz) *
                           b2g_pow(CD[0], ed[0] - dx) * b2g_pow(CD[1], ed[1] - dy) * b2g_pow(CD[2], ed[2] - dz);
              const int jf = b2g_cidx(ec[0] + dx, ec[1] + dy, ec[2] + dz);
              s += cb * cd * acc[w][ie][jf];
            }
      }
  return s;
}

// Cartesian exponents of component k of a shell with l <= 1 (s; p_x, p_y, p_z)
B2_HD void b2g_comp(int l, int k, int *e) {
  e[0] = e[1] = e[2] = 0;
  if (l) e[k] = 1;
}

// Gradient contributions of the shell quartet (a b | c d) of class (LA LB | LC LD) contracted
// with gam[ia][ib][ic][id] (component order of each shell, flattened): g[s][x] = sum gam
// d(ab|cd)/dR_x of the centre of shell s (s = 0..3; the fourth from translation invariance).
template <typename T, int LA, int LB, int LC, int LD>
B2_HD void b2g_quartet_grad_t(const B2Shell &a, const B2Shell &b, const B2Shell &c, const B2Shell &d,
                              const T *btab, const T *gam, T g[4][3]) {
  constexpr int na = 2 * LA + 1, nb = 2 * LB + 1, nc = 2 * LC + 1, nd = 2 * LD + 1;
  constexpr int LEB = LA + LB + 1, LFB = LC + LD, LEK = LA + LB, LFK = LC + LD + 1;
  T accB[3][b2g_ncart(LEB)][b2g_ncart(LFB)], accK[2][b2g_ncart(LEK)][b2g_ncart(LFK)];
  b2g_e0f0<T, LEB, LFB, false>(a, b, c, d, btab, accB);   // bra raised by one (dA, dB)
  b2g_e0f0<T, LEK, LFK, true>(a, b, c, d, btab, accK);    // ket raised by one (dC)
  T AB[3], CD[3];
  for (int x = 0; x < 3; ++x) {
    AB[x] = (T)(a.R[x] - b.R[x]);
    CD[x] = (T)(c.R[x] - d.R[x]);
  }
  for (int s = 0; s < 4; ++s) for (int x = 0; x < 3; ++x) g[s][x] = (T)0;
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib)
      for (int ic = 0; ic < nc; ++ic)
        for (int id = 0; id < nd; ++id) {
          const T gm = gam[((ia * nb + ib) * nc + ic) * nd + id];
          if (gm == (T)0) continue;
          int ea[3], eb[3], ec[3], ed[3];
          b2g_comp(LA, ia, ea); b2g_comp(LB, ib, eb); b2g_comp(LC, ic, ec); b2g_comp(LD, id, ed);
          for (int x = 0; x < 3; ++x) {
            int up[3], dn[3];
            // d/dA_x: 2 alpha (a+1x b| - a_x (a-1x b|
            for (int k = 0; k < 3; ++k) { up[k] = ea[k] + (k == x); dn[k] = ea[k] - (k == x); }
            T dA = b2g_hrr(accB, 1, up, eb, ec, ed, AB, CD);
            if (ea[x]) dA -= (T)ea[x] * b2g_hrr(accB, 0, dn, eb, ec, ed, AB, CD);
            // d/dB_x: 2 beta (a b+1x| - b_x (a b-1x|
            for (int k = 0; k < 3; ++k) { up[k] = eb[k] + (k == x); dn[k] = eb[k] - (k == x); }
            T dB = b2g_hrr(accB, 2, ea, up, ec, ed, AB, CD);
            if (eb[x]) dB -= (T)eb[x] * b2g_hrr(accB, 0, ea, dn, ec, ed, AB, CD);
            // d/dC_x: 2 gamma (ab|c+1x d) - c_x (ab|c-1x d)
            for (int k = 0; k < 3; ++k) { up[k] = ec[k] + (k == x); dn[k] = ec[k] - (k == x); }
            T dC = b2g_hrr(accK, 1, ea, eb, up, ed, AB, CD);
            if (ec[x]) dC -= (T)ec[x] * b2g_hrr(accK, 0, ea, eb, dn, ed, AB, CD);
            g[0][x] += gm * dA;
            g[1][x] += gm * dB;
            g[2][x] += gm * dC;
          }
        }
  for (int x = 0; x < 3; ++x) g[3][x] = -(g[0][x] + g[1][x] + g[2][x]);
}

// the same for shells of any class (l <= 1), dispatched at run time
template <typename T>
B2_HD void b2g_quartet_grad(const B2Shell &a, const B2Shell &b, const B2Shell &c, const B2Shell &d,
                            const T *btab, const T *gam, T g[4][3]) {
  switch (a.l * 8 + b.l * 4 + c.l * 2 + d.l) {
#define B2G_Q(A, B, C, D) case A * 8 + B * 4 + C * 2 + D: b2g_quartet_grad_t<T, A, B, C, D>(a, b, c, d, btab, gam, g); break;
    B2G_Q(0, 0, 0, 0) B2G_Q(0, 0, 0, 1) B2G_Q(0, 0, 1, 0) B2G_Q(0, 0, 1, 1)
    B2G_Q(0, 1, 0, 0) B2G_Q(0, 1, 0, 1) B2G_Q(0, 1, 1, 0) B2G_Q(0, 1, 1, 1)
    B2G_Q(1, 0, 0, 0) B2G_Q(1, 0, 0, 1) B2G_Q(1, 0, 1, 0) B2G_Q(1, 0, 1, 1)
    B2G_Q(1, 1, 0, 0) B2G_Q(1, 1, 0, 1) B2G_Q(1, 1, 1, 0) B2G_Q(1, 1, 1, 1)
#undef B2G_Q
    default: break;
  }
}

// Work-list group g = bra class * 4 + ket class (class = l_first + 2 l_second) to the shells'
// angular momenta: k = 0..3 gives l of I, J, K, L.
B2_HD constexpr int b2g_group_l(int g, int k) {
  return k == 0 ? (g >> 2) & 1 : k == 1 ? (g >> 3) & 1 : k == 2 ? g & 1 : (g >> 1) & 1;
}

// One canonical shell quartet (a b | c d) (pair index IJ >= KL, I >= J, K >= L) of a molecule
// with density Dm (N x N): summed over all ordered index quartets, dE_2e/dR = sum d(ij|kl)/dR
// Gamma_ijkl, Gamma = 1/2 D_ij D_kl - hyb/4 D_il D_jk; over the eight orderings of a quartet
// that is the symmetrised Gamma = 1/2 D_ij D_kl - hyb/8 (D_il D_jk + D_ik D_jl) times the number
// of distinct shell orderings (2 for I != J, 2 for K != L, 2 for IJ != KL).
template <int LA, int LB, int LC, int LD>
B2_HD void b2g_canonical_quartet(const B2Shell &a, const B2Shell &b, const B2Shell &c, const B2Shell &d,
                                 bool ij_same, bool kl_same, bool braket_same, const double *Dm, int N,
                                 double hyb, const double *btab, double g4[4][3]) {
  constexpr int na = 2 * LA + 1, nb = 2 * LB + 1, nc = 2 * LC + 1, nd = 2 * LD + 1;
  const double deg = (ij_same ? 1.0 : 2.0) * (kl_same ? 1.0 : 2.0) * (braket_same ? 1.0 : 2.0);
  double gam[na * nb * nc * nd];
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib)
      for (int ic = 0; ic < nc; ++ic)
        for (int id = 0; id < nd; ++id) {
          const int i = a.ao0 + ia, j = b.ao0 + ib, k = c.ao0 + ic, l = d.ao0 + id;
          gam[((ia * nb + ib) * nc + ic) * nd + id] =
              deg * (0.5 * Dm[i * N + j] * Dm[k * N + l] -
                     0.125 * hyb * (Dm[i * N + l] * Dm[j * N + k] + Dm[i * N + k] * Dm[j * N + l]));
        }
  b2g_quartet_grad_t<double, LA, LB, LC, LD>(a, b, c, d, btab, gam, g4);
}

// ---------------------------------------------------------------- one-electron part
// d/dR of <D, T + V_nuc> - <W, S> at fixed D and W (the h1aos and s1 terms of the reference's
// grad_elec, nanoDFT.py:414-424), per ordered shell pair (a, b): overlap and kinetic integrals
// from Obara-Saika one-dimensional overlap tables (kinetic energy by the Laplacian acting on the
// ket function), nuclear attraction by the Obara-Saika vertical recursion in (a|1/r_C|0) and the
// same binomial horizontal recursion as above; the derivative with respect to a nucleus C
// follows from translation invariance of <a|1/|r - C||b>.

// 1D overlap factors s[i][j] (up to 2 x 4) of a primitive pair: i on centre A, j on centre B
template <typename T>
B2_HD void b2g_ovl1d(T PA, T PB, T oz, int ni, int nj, T s[3][5]) {
  s[0][0] = (T)1;
  for (int i = 1; i <= ni; ++i) s[i][0] = PA * s[i - 1][0] + (i > 1 ? (T)(i - 1) * oz * s[i - 2][0] : (T)0);
  for (int j = 1; j <= nj; ++j)
    for (int i = 0; i <= ni; ++i)
      s[i][j] = PB * s[i][j - 1] + oz * ((i > 0 ? (T)i * s[i - 1][j - 1] : (T)0) +
                                         (j > 1 ? (T)(j - 1) * s[i][j - 2] : (T)0));
}

// g[0], g[1]: gradient on the centres of a and b; the terms on the nuclei go to addC(atom, x,
// value) (the caller's accumulator: a plain sum on the host, atomics on the GPU).
// D and W are the molecule's nao x nao matrices (row-major, stride N); Z / RC the nuclei.
template <typename T, typename AddC>
B2_HD void b2g_pair_grad_1e(const B2Shell &a, const B2Shell &b, const T *D, const T *Wm, int N, int natm,
                            const T *Z, const T *RC, const T *btab, T g[2][3], AddC &&addC) {
  const int la = a.l, lb = b.l, na = 2 * la + 1, nb = 2 * lb + 1;
  T AB[3], AB2 = 0;
  for (int x = 0; x < 3; ++x) { AB[x] = (T)(a.R[x] - b.R[x]); AB2 += AB[x] * AB[x]; }
  for (int s = 0; s < 2; ++s) for (int x = 0; x < 3; ++x) g[s][x] = (T)0;
  // nuclear attraction: contracted Theta[w][e], e up to la + lb + 1, per nucleus
  const int le = la + lb + 1, ne = b2g_ncart(le);
  for (int pa = 0; pa < a.nprim; ++pa)
    for (int pb = 0; pb < b.nprim; ++pb) {
      const T al = (T)a.exp[pa], be = (T)b.exp[pb], z = al + be, oz = (T)0.5 / z;
      T P[3], PA[3], PB[3];
      for (int x = 0; x < 3; ++x) {
        P[x] = (al * (T)a.R[x] + be * (T)b.R[x]) / z;
        PA[x] = P[x] - (T)a.R[x];
        PB[x] = P[x] - (T)b.R[x];
      }
      const T cab = (T)a.coef[pa] * (T)b.coef[pb] * exp(-al * be / z * AB2);
      const T pref3 = cab * pow((T)3.141592653589793 / z, (T)1.5);
      T s1[3][3][5];
      for (int x = 0; x < 3; ++x) b2g_ovl1d<T>(PA[x], PB[x], oz, la + 1, lb + 3, s1[x]);
      auto S3 = [&](const int *ea, const int *eb) -> T {
        return pref3 * s1[0][ea[0]][eb[0]] * s1[1][ea[1]][eb[1]] * s1[2][ea[2]][eb[2]];
      };
      auto T3 = [&](const int *ea, const int *eb) -> T {   // -1/2 <a| lap |b>
        T t = 0;
        for (int x = 0; x < 3; ++x) {
          int e2[3] = {eb[0], eb[1], eb[2]};
          T u = -(T)2 * be * (T)(2 * eb[x] + 1) * S3(ea, eb);
          e2[x] = eb[x] + 2;
          u += (T)4 * be * be * S3(ea, e2);
          if (eb[x] >= 2) { e2[x] = eb[x] - 2; u += (T)(eb[x] * (eb[x] - 1)) * S3(ea, e2); }
          t += u;
        }
        return (T)-0.5 * t;
      };
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib) {
          int ea[3], eb[3];
          b2g_comp(la, ia, ea);
          b2g_comp(lb, ib, eb);
          const int i = a.ao0 + ia, j = b.ao0 + ib;
          const T dij = D[i * N + j], wij = Wm[i * N + j];
          for (int x = 0; x < 3; ++x) {
            int up[3] = {ea[0], ea[1], ea[2]}, dn[3] = {ea[0], ea[1], ea[2]};
            up[x]++; dn[x]--;
            T dS = (T)2 * al * S3(up, eb), dT = (T)2 * al * T3(up, eb);
            if (ea[x]) { dS -= (T)ea[x] * S3(dn, eb); dT -= (T)ea[x] * T3(dn, eb); }
            g[0][x] += dij * dT - wij * dS;
            int ub[3] = {eb[0], eb[1], eb[2]}, db[3] = {eb[0], eb[1], eb[2]};
            ub[x]++; db[x]--;
            dS = (T)2 * be * S3(ea, ub); dT = (T)2 * be * T3(ea, ub);
            if (eb[x]) { dS -= (T)eb[x] * S3(ea, db); dT -= (T)eb[x] * T3(ea, db); }
            g[1][x] += dij * dT - wij * dS;
          }
        }
      // nuclear attraction, nucleus by nucleus
      for (int c = 0; c < natm; ++c) {
        T PC[3], PC2 = 0;
        for (int x = 0; x < 3; ++x) { PC[x] = P[x] - RC[3 * c + x]; PC2 += PC[x] * PC[x]; }
        T F[B2G_MMAX];
        b2g_boys<T>(le, z * PC2, btab, F);
        T th[B2G_NC][B2G_MMAX];
        const T p0 = -Z[c] * (T)6.283185307179586 / z * cab;
        for (int m = 0; m <= le; ++m) th[0][m] = p0 * F[m];
        for (int l1 = 1; l1 <= le; ++l1)
          for (int ie = b2g_cstart(l1); ie < b2g_cstart(l1 + 1); ++ie) {
            int ex, ey, ez;
            b2g_cart(ie, ex, ey, ez);
            const int dd = ex ? 0 : (ey ? 1 : 2);
            int e1[3] = {ex, ey, ez};
            e1[dd]--;
            const int i1 = b2g_cidx(e1[0], e1[1], e1[2]);
            int i2 = -1;
            if (e1[dd] > 0) {
              int e2[3] = {e1[0], e1[1], e1[2]};
              e2[dd]--;
              i2 = b2g_cidx(e2[0], e2[1], e2[2]);
            }
            for (int m = 0; m <= le - l1; ++m) {
              T t = PA[dd] * th[i1][m] - PC[dd] * th[i1][m + 1];
              if (i2 >= 0) t += (T)e1[dd] * oz * (th[i2][m] - th[i2][m + 1]);
              th[ie][m] = t;
            }
          }
        auto V3 = [&](const int *ea, const int *eb) -> T {    // binomial horizontal recursion
          T s = 0;
          for (int bx = 0; bx <= eb[0]; ++bx)
            for (int by = 0; by <= eb[1]; ++by)
              for (int bz = 0; bz <= eb[2]; ++bz)
                s += (T)(b2g_binom(eb[0], bx) * b2g_binom(eb[1], by) * b2g_binom(eb[2], bz)) *
                     b2g_pow(AB[0], eb[0] - bx) * b2g_pow(AB[1], eb[1] - by) * b2g_pow(AB[2], eb[2] - bz) *
                     th[b2g_cidx(ea[0] + bx, ea[1] + by, ea[2] + bz)][0];
          return s;
        };
        for (int ia = 0; ia < na; ++ia)
          for (int ib = 0; ib < nb; ++ib) {
            int ea[3], eb[3];
            b2g_comp(la, ia, ea);
            b2g_comp(lb, ib, eb);
            const T dij = D[(a.ao0 + ia) * N + b.ao0 + ib];
            for (int x = 0; x < 3; ++x) {
              int up[3] = {ea[0], ea[1], ea[2]}, dn[3] = {ea[0], ea[1], ea[2]};
              up[x]++; dn[x]--;
              T dA = (T)2 * al * V3(up, eb);
              if (ea[x]) dA -= (T)ea[x] * V3(dn, eb);
              int ub[3] = {eb[0], eb[1], eb[2]}, db[3] = {eb[0], eb[1], eb[2]};
              ub[x]++; db[x]--;
              T dB = (T)2 * be * V3(ea, ub);
              if (eb[x]) dB -= (T)eb[x] * V3(ea, db);
              g[0][x] += dij * dA;
              g[1][x] += dij * dB;
              addC(c, x, -dij * (dA + dB));
            }
          }
      }
    }
}

// ---------------------------------------------------------------- exchange-correlation part
// d/dR of E_xc at fixed D on a fixed grid (the V_xc terms of the reference's grad_elec,
// nanoDFT.py:408-415; the grid does not move with the atoms, as there).  Moving atom A moves its
// orbitals (d phi_i / dR_A = -grad phi_i), so with u = D phi, u_k = D d_k phi, g = grad rho:
//   dE/dR_A,x = -2 sum_g w sum_{i on A} [vrho d_x phi_i u_i
//                                        + 2 vgamma sum_k g_k (d_x d_k phi_i u_i + d_x phi_i u_k,i)]

// values, gradients and Hessians (xx, xy, xz, yy, yz, zz) of the components of shell S at r
template <typename T>
B2_HD void b2g_ao2(const B2Shell &S, const T *r, T *f, T (*df)[3], T (*hf)[6]) {
  T d[3], r2 = 0;
  for (int x = 0; x < 3; ++x) { d[x] = r[x] - (T)S.R[x]; r2 += d[x] * d[x]; }
  T g0 = 0, g1 = 0, g2 = 0;                    // sum c e, sum c (-2a) e, sum c 4a^2 e
  for (int k = 0; k < S.nprim; ++k) {
    const T al = (T)S.exp[k], e = (T)S.coef[k] * exp(-al * r2);
    g0 += e;
    g1 += (T)-2 * al * e;
    g2 += (T)4 * al * al * e;
  }
  const int hk[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  if (S.l == 0) {
    f[0] = g0;
    for (int x = 0; x < 3; ++x) df[0][x] = g1 * d[x];
    for (int h = 0; h < 6; ++h) {
      const int p = hk[h][0], q = hk[h][1];
      hf[0][h] = g2 * d[p] * d[q] + (p == q ? g1 : (T)0);
    }
    return;
  }
  for (int c = 0; c < 3; ++c) {
    f[c] = d[c] * g0;
    for (int x = 0; x < 3; ++x) df[c][x] = (x == c ? g0 : (T)0) + d[c] * d[x] * g1;
    for (int h = 0; h < 6; ++h) {
      const int p = hk[h][0], q = hk[h][1];
      hf[c][h] = (p == c ? g1 * d[q] : (T)0) + (q == c ? g1 * d[p] : (T)0) +
                 d[c] * ((p == q ? g1 : (T)0) + d[p] * d[q] * g2);
    }
  }
}
