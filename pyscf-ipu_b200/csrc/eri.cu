// s8 ERI generator kernel (sm_100a).  Replaces the reference's per-quartet IPU vertex
// ``poplar_int2e_sph_forloop`` (int2e_sph.cpp:7180-7254) driven by ``integrals_v1``
// (direct.py:584-707), and writes straight into the tril-of-tril s8 layout of
// ``mol.intor('int2e_sph', aosym='s8')`` (nanoDFT.py:285).
//
// Decomposition: one CTA per AO-pair row ij of one molecule (rows of all molecules of
// the batch are concatenated; the CTA finds its molecule by binary search).  The CTA
// folds the row's bra components into its 9 bra primitive pairs in shared memory; its
// threads then walk the ket shell pairs KL <= IJ class by class (ss, ps, sp, pp), so a
// warp runs one specialised code path, and each thread evaluates all components of its
// ket shell pair against the row's bra AO pair.
#include "eri_row.cuh"
#include "device_plan.cuh"

template <typename T>
__global__ void __launch_bounds__(128)
k_eri_s8(const B2MolDev *__restrict__ mols, const long long *__restrict__ row_off, int nmol,
         long long row_begin, const B2PairInfo *__restrict__ pinfo,
         const B2PairPrim<T> *__restrict__ pp, const int *__restrict__ ao2sh,
         const int *__restrict__ cls_list, const int *__restrict__ cls_cnt,
         const double *__restrict__ btab, T *__restrict__ out) {
  __shared__ B2BraPrim<T> sbra[B2_MAXPP];
  __shared__ int s_nb;
  const long long row = row_begin + blockIdx.x;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {                           // last m with row_off[m] <= row
    int mid = (lo + hi + 1) >> 1;
    if (row_off[mid] <= row) lo = mid; else hi = mid - 1;
  }
  const B2MolDev md = mols[lo];
  const B2RowInfo r = b2_row_info(md, row - row_off[lo], ao2sh, pinfo);
  if (threadIdx.x == 0) {
    int nb = 0;
    const B2PairPrim<T> *bp = pp + (size_t)(md.sp_off + r.sp) * B2_MAXPP;
    for (int x = 0; x < B2_MAXPP; ++x)
      if (bp[x].K != (T)0) b2_make_bra_dispatch<T>(r.bcls, bp[x], r.ci, r.cj, sbra[nb++]);
    s_nb = nb;
  }
  __syncthreads();
  const int nb = s_nb;
  int cnt[4], pre[5];
  pre[0] = 0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    cnt[c] = cls_cnt[4ll * md.sp_off + (long long)c * md.nsp + r.spcut];
    pre[c + 1] = pre[c] + cnt[c];
  }
  T *out_mol = out + md.eri_off;
  for (int t = threadIdx.x; t < pre[4]; t += blockDim.x) {
    int c = (t >= pre[1]) + (t >= pre[2]) + (t >= pre[3]);
    int KL = cls_list[md.sp_off + md.cls_start[c] + (t - pre[c])];
    const B2PairInfo kp = pinfo[md.sp_off + KL];
    T acc[3][3];
    b2_eri_dispatch<T>(r.bcls, c, sbra, nb, pp + (size_t)(md.sp_off + KL) * B2_MAXPP, r.ci, r.cj,
                       btab, acc);
    b2_eri_store<T, T>(out_mol, r.ij, kp, kp.I == kp.J, acc);
  }
}

int b2_launch_eri_s8(const B2PlanDev &P, int precision, void *out, cudaStream_t st) {
  const long long chunk = 1ll << 30;
  for (long long r0 = 0; r0 < P.h.n_rows; r0 += chunk) {
    unsigned nblk = (unsigned)std::min(chunk, P.h.n_rows - r0);
    if (precision == 64)
      k_eri_s8<double><<<nblk, 128, 0, st>>>(P.mols, P.row_off, P.h.nmol, r0, P.pinfo, P.pp64,
                                             P.ao2sh, P.cls_list, P.cls_cnt, P.boys,
                                             (double *)out);
    else if (precision == 32)
      k_eri_s8<float><<<nblk, 128, 0, st>>>(P.mols, P.row_off, P.h.nmol, r0, P.pinfo, P.pp32,
                                            P.ao2sh, P.cls_list, P.cls_cnt, P.boys, (float *)out);
    else
      return B2_ERR_ARG;
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
