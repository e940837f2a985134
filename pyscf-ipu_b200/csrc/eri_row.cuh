// Shared row logic of the s8 ERI generator: one bra AO pair ij (a "row" of the packed
// (ij|kl) matrix, kl <= ij) against every ket shell pair KL <= IJ, grouped by angular class.
#pragma once
#include "eri_math.cuh"
#include "plan_host.hpp"

template <typename T, int LI, int LJ>
B2_HD void b2_eri_ket(int cls, const B2BraPrim<T> *bra, int nb, const B2PairPrim<T> *ket, int ci,
                      int cj, const double *btab, T acc[3][3]) {
  switch (cls) {
    case 0: b2_eri_item<T, LI, LJ, 0, 0>(bra, nb, ket, B2_MAXPP, ci, cj, btab, acc); break;
    case 1: b2_eri_item<T, LI, LJ, 1, 0>(bra, nb, ket, B2_MAXPP, ci, cj, btab, acc); break;
    case 2: b2_eri_item<T, LI, LJ, 0, 1>(bra, nb, ket, B2_MAXPP, ci, cj, btab, acc); break;
    default: b2_eri_item<T, LI, LJ, 1, 1>(bra, nb, ket, B2_MAXPP, ci, cj, btab, acc); break;
  }
}

template <typename T>
B2_HD void b2_eri_dispatch(int bcls, int cls, const B2BraPrim<T> *bra, int nb,
                           const B2PairPrim<T> *ket, int ci, int cj, const double *btab,
                           T acc[3][3]) {
  switch (bcls) {
    case 0: b2_eri_ket<T, 0, 0>(cls, bra, nb, ket, ci, cj, btab, acc); break;
    case 1: b2_eri_ket<T, 1, 0>(cls, bra, nb, ket, ci, cj, btab, acc); break;
    case 2: b2_eri_ket<T, 0, 1>(cls, bra, nb, ket, ci, cj, btab, acc); break;
    default: b2_eri_ket<T, 1, 1>(cls, bra, nb, ket, ci, cj, btab, acc); break;
  }
}

template <typename T>
B2_HD void b2_make_bra_dispatch(int bcls, const B2PairPrim<T> &P, int ci, int cj, B2BraPrim<T> &B) {
  switch (bcls) {
    case 0: b2_make_bra<T, 0, 0>(P, ci, cj, B); break;
    case 1: b2_make_bra<T, 1, 0>(P, ci, cj, B); break;
    case 2: b2_make_bra<T, 0, 1>(P, ci, cj, B); break;
    default: b2_make_bra<T, 1, 1>(P, ci, cj, B); break;
  }
}

// store the ket block of row ij into the s8 list of one molecule
template <typename T, typename TO>
B2_HD void b2_eri_store(TO *out_mol, long long ij, const B2PairInfo &kp, bool same_shell,
                        const T acc[3][3]) {
  const int nk = 2 * kp.lI + 1, nl = 2 * kp.lJ + 1;
  const long long rowbase = b2_tri(ij);
  for (int ck = 0; ck < nk; ++ck)
    for (int cl = 0; cl < nl; ++cl) {
      int k = kp.ao0I + ck, l = kp.ao0J + cl;
      if (same_shell && l > k) continue;
      long long kl = b2_tri(k) + l;
      if (kl > ij) continue;
      out_mol[rowbase + kl] = (TO)acc[ck][cl];
    }
}

// bra set-up of one row: molecule-local AO indices -> shells, components, bra class
struct B2RowInfo {
  long long ij;
  int i, j, I, J, ci, cj, sp, bcls;
  int spcut;   // ket shell pairs KL <= spcut = (I,I) can hold AO pairs kl <= ij
};

B2_HD B2RowInfo b2_row_info(const B2MolDev &md, long long ij, const int *ao2sh, const B2PairInfo *pinfo) {
  B2RowInfo r;
  r.ij = ij;
  r.i = (int)b2_untri(ij);
  r.j = (int)(ij - b2_tri(r.i));
  r.I = ao2sh[md.ao_off + r.i];
  r.J = ao2sh[md.ao_off + r.j];
  r.sp = (int)b2_tri(r.I) + r.J;
  const B2PairInfo &pi = pinfo[md.sp_off + r.sp];
  r.ci = r.i - pi.ao0I;
  r.cj = r.j - pi.ao0J;
  r.bcls = pi.lI + 2 * pi.lJ;
  r.spcut = (int)b2_tri(r.I) + r.I;
  return r;
}
