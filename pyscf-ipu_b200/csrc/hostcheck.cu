// Test-only host build of the device math (ERI shell quartets, Boys function, B3LYP point
// functional, gradient terms).  It runs the exact __host__ __device__ code the kernels run, on the CPU, so
// the CPU test suite can check the kernel arithmetic against the oracle without a GPU.
// It is never loaded by the product path (libb200dft.so has no CPU fallback).
#include "eri_sq.cuh"
#include "grad_math.cuh"
#include "xc_math.cuh"
#include <algorithm>
#include <vector>

// The two-electron gradient kernels' traversal on the host: the float32 ERI work list (32 kets
// per task, grouped by class combination), canonical quartets only, each quartet through the
// serial b2g_canonical_quartet with the class its group fixes (the GPU kernels split the same
// recursions over a warp's lanes; b2hc_grad_vrr_tables checks their step tables).  bad counts
// quartets whose shells do not have the group's angular momenta.
template <int G>
static void b2hc_2e_group(const B2PlanHost &P, const std::vector<B2EriTask> &tasks, const std::vector<long long> &goff,
                          const double *D, double hyb, const double *tab, double *g, int *bad) {
  for (long long t = goff[G]; t < goff[G + 1]; ++t) {
    const B2EriTask &tk = tasks[t];
    const B2MolDev &md = P.mols[tk.mol];
    const B2PairInfo &bp = P.pinfo[md.sp_off + tk.IJ];
    const B2Shell *S = &P.shells[md.sh_off];
    for (int lane = 0; lane < 32; ++lane) {
      if (lane >= tk.count) continue;
      const int KL = P.cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + lane];
      if (KL > tk.IJ) continue;
      const B2PairInfo &kp = P.pinfo[md.sp_off + KL];
      const B2Shell *q[4] = {&S[bp.I], &S[bp.J], &S[kp.I], &S[kp.J]};
      for (int k = 0; k < 4; ++k)
        if (q[k]->l != b2g_group_l(G, k)) ++*bad;
      double g4[4][3];
      b2g_canonical_quartet<b2g_group_l(G, 0), b2g_group_l(G, 1), b2g_group_l(G, 2), b2g_group_l(G, 3)>(
          *q[0], *q[1], *q[2], *q[3], bp.I == bp.J, kp.I == kp.J, KL == tk.IJ, D + md.mat_off, md.nao, hyb,
          tab, g4);
      for (int s = 0; s < 4; ++s)
        for (int x = 0; x < 3; ++x) g[3 * (md.atm_off + q[s]->atom) + x] += g4[s][x];
    }
  }
  if constexpr (G < 15) b2hc_2e_group<G + 1>(P, tasks, goff, D, hyb, tab, g, bad);
}

// The GPU kernels' tabulated vertical recursion (B2gVrr, grad_math.cuh) run on the host: every
// step of the table in order (an order the kernels' level-by-level lane split respects), summed
// over the quartet's primitive quartets with the kernels' weights, against the serial b2g_e0f0
// of the same quartet.  Returns the largest difference relative to max |entry|.
template <int LE, int LF, bool KET>
static double b2hc_vrr_table(const B2Shell &a, const B2Shell &b, const B2Shell &c, const B2Shell &d,
                             const double *tab) {
  using S = B2gVrr<LE, LF, LE + LF>;
  constexpr int L = LE + LF, NW = KET ? 2 : 3;
  double ser[NW][S::NE][S::NF];
  b2g_e0f0<double, LE, LF, KET>(a, b, c, d, tab, ser);
  std::vector<double> acc(NW * S::NACC, 0.0), v(S::NV, 0.0);
  double AB2 = 0, CD2 = 0;
  for (int x = 0; x < 3; ++x) {
    AB2 += (a.R[x] - b.R[x]) * (a.R[x] - b.R[x]);
    CD2 += (c.R[x] - d.R[x]) * (c.R[x] - d.R[x]);
  }
  for (int pa = 0; pa < a.nprim; ++pa)
    for (int pb = 0; pb < b.nprim; ++pb) {
      const double al = a.exp[pa], be = b.exp[pb], z = al + be;
      double P[3], PA[3];
      for (int x = 0; x < 3; ++x) {
        P[x] = (al * a.R[x] + be * b.R[x]) / z;
        PA[x] = P[x] - a.R[x];
      }
      const double Kab = exp(-al * be / z * AB2) * a.coef[pa] * b.coef[pb];
      for (int pc = 0; pc < c.nprim; ++pc)
        for (int pd = 0; pd < d.nprim; ++pd) {
          const double ga = c.exp[pc], de = d.exp[pd], e = ga + de;
          double Q[3], QC[3], WP[3], WQ[3], PQ2 = 0;
          for (int x = 0; x < 3; ++x) {
            Q[x] = (ga * c.R[x] + de * d.R[x]) / e;
            QC[x] = Q[x] - c.R[x];
            const double W = (z * P[x] + e * Q[x]) / (z + e);
            WP[x] = W - P[x];
            WQ[x] = W - Q[x];
            PQ2 += (P[x] - Q[x]) * (P[x] - Q[x]);
          }
          const double rho = z * e / (z + e);
          const double Kcd = exp(-ga * de / e * CD2) * c.coef[pc] * d.coef[pd];
          const double pref = 34.98683665524972 / (z * e * sqrt(z + e)) * Kab * Kcd;
          double F[L + 1];
          b2_boys<double, L, double>(rho * PQ2, tab, F);
          std::fill(v.begin(), v.end(), 0.0);
          for (int m = 0; m <= L; ++m) v[m] = pref * F[m];
          const double hb = 0.5 / z, rb = rho / z, hk = 0.5 / e, rk = rho / e, h3 = 0.5 / (z + e);
          for (int o = 0; o < S::NOP; ++o) {
            const B2gOp op = S::op(o);
            if (op.mmax < 0) continue;
            const bool bra = o < S::NOB;
            const double X = bra ? PA[op.dd] : QC[op.dd], Y = bra ? WP[op.dd] : WQ[op.dd];
            const double cc = (double)op.c1 * (bra ? hb : hk), r = bra ? rb : rk, c3 = (double)op.c3 * h3;
            for (int m = 0; m <= op.mmax; ++m) {
              double t = X * v[op.s1 + m] + Y * v[op.s1 + m + 1];
              if (op.s2 >= 0) t += cc * (v[op.s2 + m] - r * v[op.s2 + m + 1]);
              if (op.s3 >= 0) t += c3 * v[op.s3 + m + 1];
              v[op.dst + m] = t;
            }
          }
          const double w[3] = {1.0, KET ? 2 * ga : 2 * al, 2 * be};
          for (int q = 0; q < NW; ++q)
            for (int t = 0; t < S::NACC; ++t) {
              const int ie = t / S::NF, jf = t % S::NF;
              acc[q * S::NACC + t] += w[q] * v[ie * S::SE + jf * S::SM];
            }
        }
    }
  double big = 0, diff = 0;
  for (int q = 0; q < NW; ++q)
    for (int ie = 0; ie < S::NE; ++ie)
      for (int jf = 0; jf < S::NF; ++jf) {
        big = std::max(big, fabs(ser[q][ie][jf]));
        diff = std::max(diff, fabs(ser[q][ie][jf] - acc[q * S::NACC + ie * S::NF + jf]));
      }
  return big > 0 ? diff / big : diff;
}

// every class combination G: both passes of the two-electron gradient (bra raised, ket raised)
// on a fixed quartet of s / p shells with the class's angular momenta
template <int G>
static void b2hc_vrr_all(const double *tab, double *rel) {
  B2Shell sh[4] = {};
  const double R[4][3] = {{0.1, -0.2, 0.3}, {1.4, 0.5, -0.6}, {-0.9, 1.1, 0.8}, {0.7, -1.3, 1.9}};
  const double ex[4][3] = {{5.0, 0.9, 0.25}, {3.1, 0.7, 0.2}, {7.2, 1.3, 0.35}, {2.2, 0.5, 0.15}};
  const double cf[4][3] = {{0.15, 0.53, 0.44}, {0.2, 0.6, 0.35}, {0.1, 0.5, 0.5}, {0.3, 0.55, 0.3}};
  for (int k = 0; k < 4; ++k) {
    sh[k].l = b2g_group_l(G, k);
    sh[k].nprim = 3;
    sh[k].atom = k;
    for (int x = 0; x < 3; ++x) sh[k].R[x] = R[k][x];
    for (int p = 0; p < 3; ++p) { sh[k].exp[p] = ex[k][p]; sh[k].coef[p] = cf[k][p]; }
  }
  constexpr int LA = b2g_group_l(G, 0), LB = b2g_group_l(G, 1), LC = b2g_group_l(G, 2), LD = b2g_group_l(G, 3);
  rel[2 * G] = b2hc_vrr_table<LA + LB + 1, LC + LD, false>(sh[0], sh[1], sh[2], sh[3], tab);
  rel[2 * G + 1] = b2hc_vrr_table<LA + LB, LC + LD + 1, true>(sh[0], sh[1], sh[2], sh[3], tab);
  if constexpr (G < 15) b2hc_vrr_all<G + 1>(tab, rel);
}

extern "C" {

int b2hc_boys(int L, double t, double *F) {
  static std::vector<double> tab;
  if (tab.empty()) { tab.resize(B2_BOYS_NT * B2_BOYS_NM); b2_boys_fill_table(tab.data()); }
  switch (L) {
    case 0: b2_boys<double, 0>(t, tab.data(), F); break;
    case 1: b2_boys<double, 1>(t, tab.data(), F); break;
    case 2: b2_boys<double, 2>(t, tab.data(), F); break;
    case 3: b2_boys<double, 3>(t, tab.data(), F); break;
    case 4: b2_boys<double, 4>(t, tab.data(), F); break;
    default: return B2_ERR_ARG;
  }
  return B2_OK;
}

// s8 ERIs of the molecules of a batch (double output), computed with precision 64 or 32
int b2hc_eri_s8(int nmol, const int *natm, const int *nbas, const int *atm, const int *bas,
                const double *env, const long long *env_off, int precision, double *out) {
  B2PlanHost P;
  int rc = b2_plan_build(P, nmol, natm, nbas, atm, bas, env, env_off);
  if (rc) return rc;
  b2_plan_fill_pairs(P);
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  long long packed = 0;                     // output: molecules' s8 lists back to back
  std::vector<long long> base(nmol);
  for (int m = 0; m < nmol; ++m) { base[m] = packed; packed += P.mols[m].n4; }
  std::vector<float> tab32(tab.begin(), tab.end());
  std::vector<B2EriTask> tasks;
  b2_eri_tasks(P, 128, precision == 64, tasks);
  for (const B2EriTask &tk : tasks) {
    const B2MolDev &md = P.mols[tk.mol];
    const B2PairInfo &bp = P.pinfo[md.sp_off + tk.IJ];
    double *om = out + base[tk.mol];
    for (int t = 0; t < tk.count; ++t) {
      const int KL = P.cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + t];
      const B2PairInfo &kp = P.pinfo[md.sp_off + KL];
      if (precision == 64) {
        B2PairPrim<double> bra[9];
        int nb = 0;
        for (int x = 0; x < 9; ++x) {
          const B2PairPrim<double> &q = P.pp64[(size_t)(md.sp_off + tk.IJ) * 9 + x];
          if (q.K != 0) bra[nb++] = q;
        }
        b2_sq_dispatch<double, double>(bp.lI + 2 * bp.lJ, tk.cls, tk.sub, bra, nb,
                                       &P.pp64[(size_t)(md.sp_off + KL) * 9], tab.data(), om, bp, kp);
      } else {
        B2PairPrim<float> bra[9];
        int nb = 0;
        for (int x = 0; x < 9; ++x) {
          const B2PairPrim<float> &q = P.pp32[(size_t)(md.sp_off + tk.IJ) * 9 + x];
          if (q.K != 0) bra[nb++] = q;
        }
        b2_sq_dispatch<float, double>(bp.lI + 2 * bp.lJ, tk.cls, tk.sub, bra, nb,
                                      &P.pp32[(size_t)(md.sp_off + KL) * 9], tab32.data(), om, bp, kp);
      }
    }
  }
  return B2_OK;
}

// B3LYP at n points (double): rho (4, n) as in the reference (rho[1:4] = half gradient)
// class starts of every molecule as the device plan computes them (from the shells' l, no pair
// tables) and as the host pair tables give them: out_fast / out_ref hold 5 ints per molecule,
// plus the pair tables' per-class inclusive counts at the last pair (must equal the class sizes)
int b2hc_plan_classes(int nmol, const int *natm, const int *nbas, const int *atm, const int *bas,
                      const double *env, const long long *env_off, int *out_fast, int *out_ref) {
  B2PlanHost F, R;
  int rc = b2_plan_build(F, nmol, natm, nbas, atm, bas, env, env_off, /*pair_tables=*/false);
  if (rc) return rc;
  if ((rc = b2_plan_build(R, nmol, natm, nbas, atm, bas, env, env_off, /*pair_tables=*/true))) return rc;
  for (int m = 0; m < nmol; ++m) {
    const B2MolDev &md = R.mols[m];
    for (int c = 0; c < 5; ++c) {
      out_fast[5 * m + c] = F.mols[m].cls_start[c];
      out_ref[5 * m + c] = md.cls_start[c];
    }
    for (int c = 0; c < 4; ++c) {                 // class sizes from the prefix counts
      const int last = md.nsp ? R.cls_cnt[4ll * md.sp_off + (long long)c * md.nsp + md.nsp - 1] : 0;
      if (last != md.cls_start[c + 1] - md.cls_start[c]) return -100 - c;
    }
  }
  return 0;
}

// two-electron gradient of one molecule at fixed density D (nao x nao): g[natm][3] =
// sum over all ordered shell quartets of d(ij|kl)/dR Gamma_ijkl, Gamma = 1/2 D_ij D_kl - hyb/4
// D_il D_jk (the two-electron part of the reference's grad_elec, nanoDFT.py:403-426)
int b2hc_grad_2e(int natm, int nbas, const int *atm, const int *bas, const double *env, const double *D,
                 double hyb, double *g) {
  B2PlanHost P;
  const long long eo = 0;
  int rc = b2_plan_build(P, 1, &natm, &nbas, atm, bas, env, &eo);
  if (rc) return rc;
  const int N = P.mols[0].nao;
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  for (int i = 0; i < 3 * natm; ++i) g[i] = 0;
  const B2Shell *S = P.shells.data();
  std::vector<double> gam(81);
  for (int I = 0; I < nbas; ++I) for (int J = 0; J < nbas; ++J)
  for (int K = 0; K < nbas; ++K) for (int L = 0; L < nbas; ++L) {
    const B2Shell *q[4] = {&S[I], &S[J], &S[K], &S[L]};
    const int n[4] = {2 * q[0]->l + 1, 2 * q[1]->l + 1, 2 * q[2]->l + 1, 2 * q[3]->l + 1};
    for (int a = 0; a < n[0]; ++a) for (int b = 0; b < n[1]; ++b)
    for (int c = 0; c < n[2]; ++c) for (int d = 0; d < n[3]; ++d) {
      const int i = q[0]->ao0 + a, j = q[1]->ao0 + b, k = q[2]->ao0 + c, l = q[3]->ao0 + d;
      gam[((a * n[1] + b) * n[2] + c) * n[3] + d] =
          0.5 * D[i * N + j] * D[k * N + l] - 0.25 * hyb * D[i * N + l] * D[j * N + k];
    }
    double g4[4][3];
    b2g_quartet_grad<double>(*q[0], *q[1], *q[2], *q[3], tab.data(), gam.data(), g4);
    for (int s = 0; s < 4; ++s)
      for (int x = 0; x < 3; ++x) g[3 * q[s]->atom + x] += g4[s][x];
  }
  return 0;
}

// two-electron gradient of a batch (D: the molecules' matrices back to back, nao x nao each;
// g: 3 per atom, molecules back to back) by the GPU kernel's traversal
int b2hc_grad_2e_tasks(int nmol, const int *natm, const int *nbas, const int *atm, const int *bas,
                       const double *env, const long long *env_off, const double *D, double hyb, double *g,
                       int *bad) {
  B2PlanHost P;
  int rc = b2_plan_build(P, nmol, natm, nbas, atm, bas, env, env_off);
  if (rc) return rc;
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  std::vector<B2EriTask> tasks;
  std::vector<long long> goff;
  b2_eri_tasks(P, 32, false, tasks, &goff);
  for (int i = 0; i < 3 * P.n_atm; ++i) g[i] = 0;
  *bad = 0;
  b2hc_2e_group<0>(P, tasks, goff, D, hyb, tab.data(), g, bad);
  return 0;
}

// one-electron gradient of one molecule at fixed D and W (nao x nao): g[natm][3] = d/dR of
// <D, T + V_nuc> - <W, S> (nuclear repulsion not included)
int b2hc_grad_1e(int natm, int nbas, const int *atm, const int *bas, const double *env, const double *D,
                 const double *W, double *g) {
  B2PlanHost P;
  const long long eo = 0;
  int rc = b2_plan_build(P, 1, &natm, &nbas, atm, bas, env, &eo);
  if (rc) return rc;
  const int N = P.mols[0].nao;
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  std::vector<double> Z(natm), RC(3 * natm);
  for (int c = 0; c < natm; ++c) {
    Z[c] = P.atom_z[c];
    for (int x = 0; x < 3; ++x) RC[3 * c + x] = P.atom_xyz[3 * c + x];
  }
  for (int i = 0; i < 3 * natm; ++i) g[i] = 0;
  const B2Shell *S = P.shells.data();
  for (int I = 0; I < nbas; ++I)
    for (int J = 0; J < nbas; ++J) {
      double g2[2][3];
      b2g_pair_grad_1e<double>(S[I], S[J], D, W, N, natm, Z.data(), RC.data(), tab.data(), g2,
                               [&](int c, int x, double v) { g[3 * c + x] += v; });
      for (int x = 0; x < 3; ++x) {
        g[3 * S[I].atom + x] += g2[0][x];
        g[3 * S[J].atom + x] += g2[1][x];
      }
    }
  return 0;
}

// exchange-correlation gradient of one molecule at fixed D on the grid (coords G x 3, w):
// g[natm][3] = dE_xc/dR with the grid held fixed (B3LYP of xc_math.cuh)
int b2hc_grad_xc(int natm, int nbas, const int *atm, const int *bas, const double *env, const double *D,
                 long long G, const double *coords, const double *w, double *g) {
  B2PlanHost P;
  const long long eo = 0;
  int rc = b2_plan_build(P, 1, &natm, &nbas, atm, bas, env, &eo);
  if (rc) return rc;
  const int N = P.mols[0].nao;
  const B2Shell *S = P.shells.data();
  std::vector<double> f(N), u(N), uk(3 * N), df(3 * N), hf(6 * N);
  std::vector<int> own(N);
  for (int s = 0; s < nbas; ++s)
    for (int c = 0; c < 2 * S[s].l + 1; ++c) own[S[s].ao0 + c] = S[s].atom;
  for (int i = 0; i < 3 * natm; ++i) g[i] = 0;
  for (long long p = 0; p < G; ++p) {
    for (int s = 0; s < nbas; ++s) {
      double ff[3], dd[3][3], hh[3][6];
      b2g_ao2<double>(S[s], coords + 3 * p, ff, dd, hh);
      for (int c = 0; c < 2 * S[s].l + 1; ++c) {
        const int i = S[s].ao0 + c;
        f[i] = ff[c];
        for (int x = 0; x < 3; ++x) df[3 * i + x] = dd[c][x];
        for (int h = 0; h < 6; ++h) hf[6 * i + h] = hh[c][h];
      }
    }
    double rho = 0, r1[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i) {
      double a = 0, b[3] = {0, 0, 0};
      for (int j = 0; j < N; ++j) {
        a += D[i * N + j] * f[j];
        for (int x = 0; x < 3; ++x) b[x] += D[i * N + j] * df[3 * j + x];
      }
      u[i] = a;
      for (int x = 0; x < 3; ++x) uk[3 * i + x] = b[x];
      rho += f[i] * a;
      for (int x = 0; x < 3; ++x) r1[x] += df[3 * i + x] * a;
    }
    const B2XcPoint<double> o = b2_b3lyp_point<double>(rho, r1[0], r1[1], r1[2]);
    const double gr[3] = {2 * r1[0], 2 * r1[1], 2 * r1[2]};       // grad rho
    const int hidx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int i = 0; i < N; ++i)
      for (int x = 0; x < 3; ++x) {
        double t = o.vrho * df[3 * i + x] * u[i];
        double q = 0;
        for (int k = 0; k < 3; ++k) q += gr[k] * (hf[6 * i + hidx[x][k]] * u[i] + df[3 * i + x] * uk[3 * i + k]);
        t += 2 * o.vgamma * q;
        g[3 * own[i] + x] -= 2 * w[p] * t;
      }
  }
  return 0;
}

int b2hc_b3lyp(int n, const double *rho, double *exc, double *vrho, double *vgamma) {
  for (int g = 0; g < n; ++g) {
    double r[4] = {rho[g], rho[n + g], rho[2 * n + g], rho[3 * n + g]};
    B2XcPoint<double> o = b2_b3lyp_point<double>(r[0], r[1], r[2], r[3]);
    exc[g] = o.exc; vrho[g] = o.vrho; vgamma[g] = o.vgamma;
  }
  return B2_OK;
}

int b2hc_b3lyp_f32(int n, const double *rho, double *exc, double *vrho, double *vgamma) {
  for (int g = 0; g < n; ++g) {
    B2XcPoint<float> o = b2_b3lyp_point<float>((float)rho[g], (float)rho[n + g], (float)rho[2 * n + g], (float)rho[3 * n + g]);
    exc[g] = o.exc; vrho[g] = o.vrho; vgamma[g] = o.vgamma;
  }
  return B2_OK;
}

// the tabulated recursion of the GPU two-electron gradient kernels against the serial one, for
// every class combination: rel[2 G] (bra raised) and rel[2 G + 1] (ket raised), each the largest
// difference relative to the largest entry
int b2hc_grad_vrr_tables(double *rel) {
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  b2hc_vrr_all<0>(tab.data(), rel);
  return 0;
}

}  // extern "C"
