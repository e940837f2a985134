// s8 ERI generator kernel (sm_100a).  Replaces the reference's per-quartet IPU vertex
// ``poplar_int2e_sph_forloop`` (int2e_sph.cpp:7180-7254) driven by ``integrals_v1``
// (direct.py:584-707), and writes straight into the tril-of-tril s8 layout of
// ``mol.intor('int2e_sph', aosym='s8')`` (nanoDFT.py:285).
//
// Decomposition: a host-built task list (plan) assigns each CTA one bra shell pair IJ of one
// molecule and up to 128 ket shell pairs KL of a single angular class (ss, ps, sp, pp), all
// with KL <= (I,I); the bra's primitive pairs are staged in shared memory and every thread
// evaluates all components of one shell quartet (float32 form) or of one bra component
// (float64 form, p bras split over 3 threads).  Every s8 entry is written exactly once, by the
// CTA whose bra shell pair owns its row ij.
#include "eri_sq.cuh"
#include "device_plan.cuh"

template <typename T, int LI, int LJ, int LK, int LL>
__global__ void __launch_bounds__(128)
k_eri_sq(const B2EriTask *__restrict__ tasks, const B2MolDev *__restrict__ mols,
         const B2PairInfo *__restrict__ pinfo, const B2PairPrim<T> *__restrict__ pp,
         const int *__restrict__ cls_list, const double *__restrict__ btab, T *__restrict__ out) {
  __shared__ B2PairPrim<T> sbra[B2_MAXPP];
  __shared__ int s_nb;
  const B2EriTask tk = tasks[blockIdx.x];
  const B2MolDev md = mols[tk.mol];
  const B2PairInfo bp = pinfo[md.sp_off + tk.IJ];
  if (threadIdx.x == 0) {
    const B2PairPrim<T> *src = pp + (size_t)(md.sp_off + tk.IJ) * B2_MAXPP;
    int nb = 0;
    for (int x = 0; x < B2_MAXPP; ++x)
      if (src[x].K != (T)0) sbra[nb++] = src[x];
    s_nb = nb;
  }
  __syncthreads();
  if ((int)threadIdx.x >= tk.count) return;
  const int KL = cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + threadIdx.x];
  const B2PairInfo kp = pinfo[md.sp_off + KL];
  b2_sq_sub<T, LI, LJ, LK, LL, T>(tk.sub, sbra, s_nb, pp + (size_t)(md.sp_off + KL) * B2_MAXPP,
                                  btab, out + md.eri_off, bp, kp);
}

template <typename T, int LI, int LJ, int LK, int LL>
static void b2_eri_group(const B2PlanDev &P, const B2EriTask *tasks, long long n,
                         const B2PairPrim<T> *pp, T *out, cudaStream_t st) {
  const long long maxg = (1ll << 31) - 1;
  for (long long t0 = 0; t0 < n; t0 += maxg)
    k_eri_sq<T, LI, LJ, LK, LL><<<(unsigned)std::min(maxg, n - t0), 128, 0, st>>>(
        tasks + t0, P.mols, P.pinfo, pp, P.cls_list, P.boys, out);
}

template <typename T>
static void b2_eri_all(const B2PlanDev &P, const B2EriTask *tasks, const std::vector<long long> &g,
                       const B2PairPrim<T> *pp, T *out, cudaStream_t st) {
#define B2_G(grp, LI, LJ, LK, LL)                                                            \
  if (g[grp + 1] > g[grp])                                                                   \
    b2_eri_group<T, LI, LJ, LK, LL>(P, tasks + g[grp], g[grp + 1] - g[grp], pp, out, st);
  B2_G(0, 0, 0, 0, 0) B2_G(1, 0, 0, 1, 0) B2_G(2, 0, 0, 0, 1) B2_G(3, 0, 0, 1, 1)
  B2_G(4, 1, 0, 0, 0) B2_G(5, 1, 0, 1, 0) B2_G(6, 1, 0, 0, 1) B2_G(7, 1, 0, 1, 1)
  B2_G(8, 0, 1, 0, 0) B2_G(9, 0, 1, 1, 0) B2_G(10, 0, 1, 0, 1) B2_G(11, 0, 1, 1, 1)
  B2_G(12, 1, 1, 0, 0) B2_G(13, 1, 1, 1, 0) B2_G(14, 1, 1, 0, 1) B2_G(15, 1, 1, 1, 1)
#undef B2_G
}

static int b2_eri_task_upload(B2PlanDev &P, int precision) {
  B2EriTask *&dst = precision == 64 ? P.eri_tasks64 : P.eri_tasks32;
  std::vector<long long> &goff = precision == 64 ? P.eri_goff64 : P.eri_goff32;
  if (dst) return B2_OK;
  std::vector<B2EriTask> t;
  b2_eri_tasks(P.h, 128, precision == 64, t, &goff);
  B2_CUDA_TRY(cudaMalloc(&dst, sizeof(B2EriTask) * std::max<size_t>(1, t.size())));
  if (!t.empty())
    B2_CUDA_TRY(cudaMemcpy(dst, t.data(), sizeof(B2EriTask) * t.size(), cudaMemcpyHostToDevice));
  return B2_OK;
}

int b2_launch_eri_s8(B2PlanDev &P, int precision, void *out, cudaStream_t st) {
  if (precision != 64 && precision != 32) return B2_ERR_ARG;
  int rc = b2_eri_task_upload(P, precision);
  if (rc) return rc;
  if (precision == 64)
    b2_eri_all<double>(P, P.eri_tasks64, P.eri_goff64, P.pp64, (double *)out, st);
  else
    b2_eri_all<float>(P, P.eri_tasks32, P.eri_goff32, P.pp32, (float *)out, st);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
