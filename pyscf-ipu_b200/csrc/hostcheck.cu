// Test-only host build of the device math (ERI row items, Boys function, B3LYP point
// functional).  It runs the exact __host__ __device__ code the kernels run, on the CPU, so
// the CPU test suite can check the kernel arithmetic against the oracle without a GPU.
// It is never loaded by the product path (libb200dft.so has no CPU fallback).
#include "eri_row.cuh"
#include "xc_math.cuh"
#include <vector>

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
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  long long packed = 0;                     // output: molecules' s8 lists back to back
  for (int m = 0; m < nmol; ++m) {
    const B2MolDev &md = P.mols[m];
    long long n2 = (long long)md.nao * (md.nao + 1) / 2;
    double *om = out + packed;
    packed += md.n4;
    for (long long ij = 0; ij < n2; ++ij) {
      B2RowInfo r = b2_row_info(md, ij, P.ao2sh.data(), P.pinfo.data());
      int cnt[4];
      for (int c = 0; c < 4; ++c) cnt[c] = P.cls_cnt[4ll * md.sp_off + (long long)c * md.nsp + r.spcut];
      if (precision == 64) {
        B2BraPrim<double> bra[9];
        int nb = 0;
        const B2PairPrim<double> *bp = &P.pp64[(size_t)(md.sp_off + r.sp) * B2_MAXPP];
        for (int x = 0; x < 9; ++x) if (bp[x].K != 0) b2_make_bra_dispatch<double>(r.bcls, bp[x], r.ci, r.cj, bra[nb++]);
        for (int c = 0; c < 4; ++c)
          for (int e = 0; e < cnt[c]; ++e) {
            int KL = P.cls_list[md.sp_off + md.cls_start[c] + e];
            const B2PairInfo &kp = P.pinfo[md.sp_off + KL];
            double acc[3][3];
            b2_eri_dispatch<double>(r.bcls, c, bra, nb, &P.pp64[(size_t)(md.sp_off + KL) * 9], r.ci, r.cj, tab.data(), acc);
            b2_eri_store<double, double>(om, ij, kp, kp.I == kp.J, acc);
          }
      } else {
        B2BraPrim<float> bra[9];
        int nb = 0;
        const B2PairPrim<float> *bp = &P.pp32[(size_t)(md.sp_off + r.sp) * B2_MAXPP];
        for (int x = 0; x < 9; ++x) if (bp[x].K != 0) b2_make_bra_dispatch<float>(r.bcls, bp[x], r.ci, r.cj, bra[nb++]);
        for (int c = 0; c < 4; ++c)
          for (int e = 0; e < cnt[c]; ++e) {
            int KL = P.cls_list[md.sp_off + md.cls_start[c] + e];
            const B2PairInfo &kp = P.pinfo[md.sp_off + KL];
            float acc[3][3];
            b2_eri_dispatch<float>(r.bcls, c, bra, nb, &P.pp32[(size_t)(md.sp_off + KL) * 9], r.ci, r.cj, tab.data(), acc);
            b2_eri_store<float, double>(om, ij, kp, kp.I == kp.J, acc);
          }
      }
    }
  }
  return B2_OK;
}

// B3LYP at n points (double): rho (4, n) as in the reference (rho[1:4] = half gradient)
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

}  // extern "C"
