// Host-side batch plan: turns the libcint atm/bas/env arrays of a batch of molecules
// (the inputs the reference packs for its ERI kernels, electron_repulsion/direct.py:710-739,
// int2e_sph.cpp:6750) into the per-molecule tables the device kernels read.
//
// Per molecule:
//   * shells (B2Shell): centre, exponents, coefficients (libcint coefficient times the
//     angular factor 1/sqrt(4pi) or sqrt(3/(4pi))), l, first AO;
//   * shell pairs I>=J, index sp = I(I+1)/2+J, each with up to 9 primitive pairs
//     (zeta, P, K, P-A, P-B); K folds c_a c_b exp(-ab/zeta |AB|^2) sqrt(2) pi^{5/4}/zeta so that
//     the primitive-quartet prefactor is K_bra K_ket / sqrt(zeta+eta);
//   * shell pairs grouped by angular class (ss, ps, sp, pp), ascending, with for every
//     bra shell pair IJ the number of class members KL <= IJ (so a row's ket work is a
//     prefix of each class list);
//   * offsets of the molecule's s8 ERI list (n2(n2+1)/2 entries, n2 = nao(nao+1)/2),
//     of its AO-pair rows and of its nao x nao matrices.
#pragma once
#include <vector>
#include <cmath>
#include <cstring>
#include <algorithm>
#include "common.cuh"

struct B2MolDev {
  int nao, nbas, natm, nocc;
  int sh_off, sp_off, ao_off, nsp;
  int cls_start[5];
  int atm_off, pad0, pad1;
  long long eri_off, row_off, mat_off, n4;
};

struct B2PlanHost {
  int nmol = 0;
  int max_nao = 0, max_nbas = 0, max_natm = 0;
  long long n_eri = 0, n_rows = 0, n_mat = 0;
  int n_sh = 0, n_sp = 0, n_ao = 0, n_atm = 0;   // n_eri: padded total (see eri_off)
  std::vector<B2MolDev> mols;
  std::vector<long long> row_off;         // nmol + 1
  std::vector<B2Shell> shells;
  std::vector<B2PairInfo> pinfo;
  std::vector<B2PairPrim<double>> pp64;   // filled by b2_plan_fill_pairs (host builds only;
  std::vector<B2PairPrim<float>> pp32;    // the device plan computes them on the GPU)
  std::vector<int> ao2sh;                 // per AO: local shell index
  std::vector<int> cls_list;              // per molecule nsp entries (offset sp_off)
  std::vector<int> cls_cnt;               // per molecule 4*nsp (offset 4*sp_off)
  std::vector<double> atom_xyz;           // per atom (offset atm_off): x,y,z
  std::vector<int> atom_z;
};

B2_HD int b2_class(int lK, int lL) { return lK + 2 * lL; }   // ss=0, ps=1, sp=2, pp=3

// primitive pair x (= ia * B2_MAXPRIM + ib) of shells a, b: zeta, centre P, P-A, P-B and
// K = c_a c_b exp(-a b / zeta |AB|^2) sqrt(2) pi^{5/4} / zeta; absent primitives give an inert
// entry (zeta 1, K 0).  Shared by the device plan kernel and the host test build.
B2_HD void b2_pair_prim(const B2Shell &a, const B2Shell &b, int x, B2PairPrim<double> &q) {
  q.zeta = 1.0; q.Px = q.Py = q.Pz = 0.0; q.K = 0.0;
  q.PAx = q.PAy = q.PAz = q.PBx = q.PBy = q.PBz = 0.0; q.h2z = 0.5;
  const int pa = x / B2_MAXPRIM, pb = x % B2_MAXPRIM;
  if (pa >= a.nprim || pb >= b.nprim) return;
  const double k0 = 5.914967172795613;           // sqrt(2) pi^(5/4)
  double AB2 = 0;
  for (int d = 0; d < 3; ++d) AB2 += (a.R[d] - b.R[d]) * (a.R[d] - b.R[d]);
  const double al = a.exp[pa], be = b.exp[pb], z = al + be;
  double Pc[3];
  for (int d = 0; d < 3; ++d) Pc[d] = (al * a.R[d] + be * b.R[d]) / z;
  double K = a.coef[pa] * b.coef[pb] * exp(-al * be / z * AB2) * k0 / z;
  if (fabs(K) < 1e-300) K = 0;
  q.zeta = z; q.Px = Pc[0]; q.Py = Pc[1]; q.Pz = Pc[2]; q.K = K; q.h2z = 0.5 / z;
  q.PAx = Pc[0] - a.R[0]; q.PAy = Pc[1] - a.R[1]; q.PAz = Pc[2] - a.R[2];
  q.PBx = Pc[0] - b.R[0]; q.PBy = Pc[1] - b.R[1]; q.PBz = Pc[2] - b.R[2];
}

B2_HD void b2_pair_prim32(const B2PairPrim<double> &q, B2PairPrim<float> &f) {
  f.zeta = (float)q.zeta; f.Px = (float)q.Px; f.Py = (float)q.Py; f.Pz = (float)q.Pz;
  f.K = (float)q.K; f.PAx = (float)q.PAx; f.PAy = (float)q.PAy; f.PAz = (float)q.PAz;
  f.PBx = (float)q.PBx; f.PBy = (float)q.PBy; f.PBz = (float)q.PBz; f.h2z = (float)q.h2z;
}

// Primitive-pair screening: a primitive pair whose prefactor |K| is below the threshold
// contributes at most |K| * max|K| / sqrt(zeta + eta) times an angular factor to any ERI of
// the pair, i.e. < 1e-12 for the float64 tables and < 1e-8 for the float32 ones, below the
// accuracy of each form (the reference drops primitive pairs below exp(-60), libcint's
// expcutoff).  Surviving pairs are packed first, so a loop over a pair's primitives can stop
// at the first inert entry (K = 0).
#define B2_PP_SCREEN64 1e-15
#define B2_PP_SCREEN32 1e-11
B2_HD void b2_pair_prims_packed(const B2Shell &a, const B2Shell &b, B2PairPrim<double> *q64,
                                B2PairPrim<float> *q32, int *n32_out = nullptr) {
  B2PairPrim<double> all[B2_MAXPP];
  for (int x = 0; x < B2_MAXPP; ++x) b2_pair_prim(a, b, x, all[x]);
  int n64 = 0, n32 = 0;
  for (int x = 0; x < B2_MAXPP; ++x) {
    const double k = fabs(all[x].K);
    if (all[x].K != 0.0 && k >= B2_PP_SCREEN64) q64[n64++] = all[x];
    if (all[x].K != 0.0 && k >= B2_PP_SCREEN32) b2_pair_prim32(all[x], q32[n32++]);
  }
  B2PairPrim<double> inert;
  b2_pair_prim(a, b, B2_MAXPP * B2_MAXPP, inert);          // out-of-range index: inert entry
  for (int x = n64; x < B2_MAXPP; ++x) q64[x] = inert;
  for (int x = n32; x < B2_MAXPP; ++x) b2_pair_prim32(inert, q32[x]);
  if (n32_out) *n32_out = n32;                              // surviving float32 primitive pairs
}

// returns B2_OK or an error code
// pair_tables: also fill pinfo / cls_list / cls_cnt here (the host test build); the device plan
// builds them with k_plan_pairs and keeps only per-molecule and per-shell work on the host.
static int b2_plan_build(B2PlanHost &P, int nmol, const int *natm, const int *nbas, const int *atm,
                         const int *bas, const double *env, const long long *env_off,
                         bool pair_tables = true) {
  P = B2PlanHost();
  P.nmol = nmol;
  P.mols.resize(nmol);
  P.row_off.assign(nmol + 1, 0);
  long long tot_sh = 0, tot_atm = 0, tot_sp = 0;
  for (int m = 0; m < nmol; ++m) {
    tot_sh += nbas[m];
    tot_atm += natm[m];
    tot_sp += (long long)nbas[m] * (nbas[m] + 1) / 2;
  }
  if (tot_sp >= (1ll << 31) / 4) return B2_ERR_SIZE;
  P.shells.reserve(tot_sh);
  P.ao2sh.reserve(3 * tot_sh);
  P.atom_xyz.reserve(3 * tot_atm);
  P.atom_z.reserve(tot_atm);
  if (pair_tables) {
    P.pinfo.reserve(tot_sp);
    P.cls_list.reserve(tot_sp);
    P.cls_cnt.reserve(4 * tot_sp);
  }
  int atm_row = 0, bas_row = 0;
  for (int m = 0; m < nmol; ++m) {
    const int *A = atm + (size_t)atm_row * B2_ATM_SLOTS;
    const int *Bs = bas + (size_t)bas_row * B2_BAS_SLOTS;
    const double *E = env + env_off[m];
    B2MolDev md;
    std::memset(&md, 0, sizeof(md));
    md.natm = natm[m];
    md.nbas = nbas[m];
    md.sh_off = P.n_sh;
    md.sp_off = P.n_sp;
    md.ao_off = P.n_ao;
    md.atm_off = P.n_atm;
    int nao = 0, nel = 0;
    for (int a = 0; a < natm[m]; ++a) {
      nel += A[a * B2_ATM_SLOTS + 0];
      const double *R = E + A[a * B2_ATM_SLOTS + B2_PTR_COORD];
      P.atom_xyz.push_back(R[0]); P.atom_xyz.push_back(R[1]); P.atom_xyz.push_back(R[2]);
      P.atom_z.push_back(A[a * B2_ATM_SLOTS + 0]);
    }
    for (int s = 0; s < nbas[m]; ++s) {
      const int *b = Bs + s * B2_BAS_SLOTS;
      int l = b[B2_ANG_OF], np = b[B2_NPRIM_OF];
      if (l > B2_MAXL || np > B2_MAXPRIM || np < 1 || b[B2_NCTR_OF] != 1) return B2_ERR_UNSUPPORTED;
      if (b[B2_ATOM_OF] < 0 || b[B2_ATOM_OF] >= natm[m]) return B2_ERR_ARG;
      B2Shell sh;
      std::memset(&sh, 0, sizeof(sh));
      const double *R = E + A[b[B2_ATOM_OF] * B2_ATM_SLOTS + B2_PTR_COORD];
      for (int d = 0; d < 3; ++d) sh.R[d] = R[d];
      double fac = l == 0 ? B2_FAC_S : B2_FAC_P;
      for (int k = 0; k < np; ++k) {
        sh.exp[k] = E[b[B2_PTR_EXP] + k];
        sh.coef[k] = E[b[B2_PTR_COEFF] + k] * fac;
      }
      sh.l = l; sh.ao0 = nao; sh.nprim = np; sh.atom = b[B2_ATOM_OF];
      for (int c = 0; c < 2 * l + 1; ++c) P.ao2sh.push_back(s);
      nao += 2 * l + 1;
      P.shells.push_back(sh);
    }
    if (nao > B2_MAXNAO - 2) return B2_ERR_SIZE;
    md.nao = nao;
    md.nocc = nel / 2;
    int nsp = nbas[m] * (nbas[m] + 1) / 2;
    md.nsp = nsp;
    long long n2 = (long long)nao * (nao + 1) / 2;
    md.n4 = n2 * (n2 + 1) / 2;
    md.eri_off = P.n_eri;
    md.row_off = P.n_rows;
    md.mat_off = P.n_mat;
    // class starts: pairs (I, J <= I) of class lI + 2 lJ, counted from the shells' l in O(nbas)
    const B2Shell *S = &P.shells[md.sh_off];
    int ccount[4] = {0, 0, 0, 0}, nl[2] = {0, 0};
    for (int I = 0; I < nbas[m]; ++I) {
      ++nl[S[I].l];
      ccount[b2_class(S[I].l, 0)] += nl[0];
      ccount[b2_class(S[I].l, 1)] += nl[1];
    }
    for (int c = 0, start = 0; c < 4; ++c) { md.cls_start[c] = start; start += ccount[c]; }
    md.cls_start[4] = nsp;
    if (pair_tables) {
      // shell pairs
      std::vector<int> cls(nsp);
      for (int I = 0; I < nbas[m]; ++I)
        for (int J = 0; J <= I; ++J) {
          const B2Shell &a = S[I], &b = S[J];
          B2PairInfo pi;
          pi.I = I; pi.J = J; pi.lI = a.l; pi.lJ = b.l; pi.ao0I = a.ao0; pi.ao0J = b.ao0;
          pi.nprim = a.nprim * b.nprim; pi.pad = 0;
          P.pinfo.push_back(pi);
          cls[(int)b2_tri(I) + J] = b2_class(a.l, b.l);
        }
      // class lists and prefix counts
      for (int c = 0; c < 4; ++c)
        for (int sp = 0; sp < nsp; ++sp)
          if (cls[sp] == c) P.cls_list.push_back(sp);
      size_t base = P.cls_cnt.size();
      P.cls_cnt.resize(base + 4 * (size_t)nsp);
      for (int c = 0; c < 4; ++c) {
        int cnt = 0;
        for (int sp = 0; sp < nsp; ++sp) {
          if (cls[sp] == c) ++cnt;
          P.cls_cnt[base + (size_t)c * nsp + sp] = cnt;
        }
      }
    }
    P.mols[m] = md;
    P.n_sh += nbas[m];
    P.n_sp += nsp;
    P.n_ao += nao;
    P.n_atm += natm[m];
    P.n_eri += (md.n4 + 31) / 32 * 32;          // 128-byte aligned per molecule (vector loads)
    P.n_rows += n2;
    P.n_mat += (long long)nao * nao;
    P.row_off[m + 1] = P.n_rows;
    P.max_nao = std::max(P.max_nao, nao);
    P.max_nbas = std::max(P.max_nbas, nbas[m]);
    P.max_natm = std::max(P.max_natm, natm[m]);
    atm_row += natm[m];
    bas_row += nbas[m];
  }
  return B2_OK;
}

// host copy of the primitive-pair tables (the device plan builds them with k_pair_prims)
static void b2_plan_fill_pairs(B2PlanHost &P) {
  P.pp64.assign((size_t)P.n_sp * B2_MAXPP, B2PairPrim<double>());
  P.pp32.assign((size_t)P.n_sp * B2_MAXPP, B2PairPrim<float>());
  for (int m = 0; m < P.nmol; ++m) {
    const B2MolDev &md = P.mols[m];
    for (int sp = 0; sp < md.nsp; ++sp) {
      const B2PairInfo &pi = P.pinfo[md.sp_off + sp];
      const size_t t = (size_t)(md.sp_off + sp) * B2_MAXPP;
      b2_pair_prims_packed(P.shells[md.sh_off + pi.I], P.shells[md.sh_off + pi.J], &P.pp64[t], &P.pp32[t]);
    }
  }
}
