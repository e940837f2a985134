// s8 ERI generator kernel (sm_100a).  Replaces the reference's per-quartet IPU vertex
// ``poplar_int2e_sph_forloop`` (int2e_sph.cpp:7180-7254) driven by ``integrals_v1``
// (direct.py:584-707), and writes straight into the tril-of-tril s8 layout of
// ``mol.intor('int2e_sph', aosym='s8')`` (nanoDFT.py:285).
//
// Decomposition: a task list (built on the device from the plan's class counts, or on the host
// for the allocation-free single-molecule entry) assigns each warp one bra shell pair IJ of one
// molecule and a chunk of ket shell pairs KL of a single angular class (ss, ps, sp, pp), all
// with KL <= (I,I) (32 kets per task for batch plans, 128 for the single-molecule entry; 4 tasks
// per CTA); the bra's primitive pairs are staged in the warp's shared-memory slot.  Batch plans
// run the float32 classes with at most 27 components in the flattened kernel k_eri_fl (lanes
// over the chunk's (ket, ket primitive pair) entries); otherwise (k_eri_sq) every lane evaluates
// all components of one shell quartet (float32) or of one bra component (float64, p bras split
// over 3 lanes), looping over the chunk's kets.  Every s8 entry is written exactly once, by the
// warp whose bra shell pair owns its row ij.
#include <type_traits>
#include "eri_sq.cuh"
#include "device_plan.cuh"
#include "devmem.cuh"
#include "eri_flops.h"

template <typename T, int LI, int LJ, int LK, int LL>
__global__ void __launch_bounds__(128)
k_eri_sq(const B2EriTask *__restrict__ tasks, long long ntask, const B2MolDev *__restrict__ mols,
         const B2PairInfo *__restrict__ pinfo, const B2PairPrim<T> *__restrict__ pp,
         const int *__restrict__ cls_list, const T *__restrict__ btab, T *__restrict__ out) {
  __shared__ B2PairPrim<T> sbra[4][B2_MAXPP];
  __shared__ int s_nb[4];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ti = (long long)blockIdx.x * 4 + w;
  if (ti >= ntask) return;                        // whole warp
  const B2EriTask tk = tasks[ti];
  const B2MolDev md = mols[tk.mol];
  const B2PairInfo bp = pinfo[md.sp_off + tk.IJ];
  if (lane == 0) {
    const B2PairPrim<T> *src = pp + (size_t)(md.sp_off + tk.IJ) * B2_MAXPP;
    int nb = 0;
    for (int x = 0; x < B2_MAXPP; ++x)
      if (src[x].K != (T)0) sbra[w][nb++] = src[x];
    s_nb[w] = nb;
  }
  __syncwarp();
  const int nb = s_nb[w];
  for (int k = lane; k < tk.count; k += 32) {
    const int KL = cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + k];
    const B2PairInfo kp = pinfo[md.sp_off + KL];
    b2_sq_sub<T, LI, LJ, LK, LL, T>(tk.sub, sbra[w], nb, pp + (size_t)(md.sp_off + KL) * B2_MAXPP,
                                    btab, out + md.eri_off, bp, kp);
  }
}

// Flattened form for the float32 classes with at most 27 components per shell quartet: the
// warp's (ket, ket primitive pair) entries are packed over the lanes (a ket's primitive pairs
// survive screening in numbers 0..9, so one ket per lane left the warp waiting for its
// largest ket); each lane sums its entry over the bra's primitive pairs, a same-ket segmented
// shuffle scan (segments <= 9 lanes, 4 steps) combines the entries of each ket in a fixed
// order, and the segment's last lane adds the sum to the ket's accumulator in shared memory.
// component block <-> flat list (unrolled: constant indices, registers only)
template <typename S>
__device__ __forceinline__ void b2_fl_flatten(const float (&acc)[S::NI][S::NJ][S::NK][S::NL], float *v) {
  int t = 0;
#pragma unroll
  for (int a = 0; a < S::NI; ++a)
#pragma unroll
    for (int b = 0; b < S::NJ; ++b)
#pragma unroll
      for (int c = 0; c < S::NK; ++c)
#pragma unroll
        for (int d = 0; d < S::NL; ++d) v[t++] = acc[a][b][c][d];
}
template <typename S>
__device__ __forceinline__ void b2_fl_unflatten(const float *v, float (&acc)[S::NI][S::NJ][S::NK][S::NL]) {
  int t = 0;
#pragma unroll
  for (int a = 0; a < S::NI; ++a)
#pragma unroll
    for (int b = 0; b < S::NJ; ++b)
#pragma unroll
      for (int c = 0; c < S::NK; ++c)
#pragma unroll
        for (int d = 0; d < S::NL; ++d) acc[a][b][c][d] = v[t++];
}

template <int LI, int LJ, int LK, int LL>
__global__ void __launch_bounds__(128)
k_eri_fl(const B2EriTask *__restrict__ tasks, long long ntask, const B2MolDev *__restrict__ mols,
         const B2PairInfo *__restrict__ pinfo, const B2PairPrim<float> *__restrict__ pp,
         const unsigned char *__restrict__ ppn, const int *__restrict__ cls_list, const float *__restrict__ btab,
         float *__restrict__ out) {
  using S = B2Sq<float, LI, LJ, LK, LL, -1>;
  constexpr int NC = S::NI * S::NJ * S::NK * S::NL;
  static_assert(NC <= 27, "flattened ERI form: at most 27 components");
  __shared__ B2PairPrim<float> sbra[4][B2_MAXPP];
  __shared__ int s_nb[4];
  __shared__ int s_off[4][32], s_kl[4][32];
  __shared__ unsigned char s_map[4][32 * B2_MAXPP];
  __shared__ float s_acc[4][32][NC];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ti = (long long)blockIdx.x * 4 + w;
  if (ti >= ntask) return;                        // whole warp
  const B2EriTask tk = tasks[ti];
  const B2MolDev md = mols[tk.mol];
  const B2PairInfo bp = pinfo[md.sp_off + tk.IJ];
  if (lane == 0) {
    const B2PairPrim<float> *src = pp + (size_t)(md.sp_off + tk.IJ) * B2_MAXPP;
    int nb = 0;
    for (int x = 0; x < B2_MAXPP; ++x)
      if (src[x].K != 0.f) sbra[w][nb++] = src[x];
    s_nb[w] = nb;
  }
  // this lane's ket (tasks of batch plans hold at most 32 kets) and its surviving primitive pairs
  int KL = 0, nq = 0;
  if (lane < tk.count) {
    KL = cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + lane];
    nq = ppn[md.sp_off + KL];
  }
  int inc = nq;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  const int E = __shfl_sync(0xffffffffu, inc, 31), exc = inc - nq;
  s_off[w][lane] = exc;
  s_kl[w][lane] = KL;
  for (int j = 0; j < nq; ++j) s_map[w][exc + j] = (unsigned char)lane;
#pragma unroll
  for (int c = 0; c < NC; ++c) s_acc[w][lane][c] = 0.f;
  __syncwarp();
  const int nb = s_nb[w];
  const B2PairPrim<float> *ppm = pp + (size_t)md.sp_off * B2_MAXPP;
  for (int e0 = 0; e0 < E; e0 += 32) {
    const int e = e0 + lane;
    const bool valid = e < E;
    const int k = valid ? (int)s_map[w][e] : -1 - lane;   // entries past the end: unique keys
    float acc[S::NI][S::NJ][S::NK][S::NL];
    S::zero(acc);
    if (valid) {
      const B2PairPrim<float> Q = ppm[(size_t)s_kl[w][k] * B2_MAXPP + (e - s_off[w][k])];
      for (int p = 0; p < nb; ++p) S::quartet(sbra[w][p], Q, btab, acc);
    }
    float a[NC];
    b2_fl_flatten<S>(acc, a);
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {                     // same-ket inclusive scan
      const int ko = __shfl_up_sync(0xffffffffu, k, o);
      const bool take = lane >= o && ko == k;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float y = __shfl_up_sync(0xffffffffu, a[c], o);
        if (take) a[c] += y;
      }
    }
    const int kn = __shfl_down_sync(0xffffffffu, k, 1);
    if (valid && (lane == 31 || kn != k))
#pragma unroll
      for (int c = 0; c < NC; ++c) s_acc[w][k][c] += a[c];
    __syncwarp();
  }
  if (lane < tk.count) {
    const B2PairInfo kp = pinfo[md.sp_off + KL];
    float acc[S::NI][S::NJ][S::NK][S::NL], a[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) a[c] = s_acc[w][lane][c];
    b2_fl_unflatten<S>(a, acc);
    S::template store<float>(out + md.eri_off, bp, kp, acc);
  }
}

template <typename T> static const T *b2_boys_table(const B2PlanDev &P);
template <> const double *b2_boys_table<double>(const B2PlanDev &P) { return P.boys; }
template <> const float *b2_boys_table<float>(const B2PlanDev &P) { return P.boys32; }

template <typename T, int LI, int LJ, int LK, int LL>
static void b2_eri_group(const B2PlanDev &P, const B2EriTask *tasks, long long n,
                         const B2PairPrim<T> *pp, T *out, cudaStream_t st) {
  const long long maxg = 4 * ((1ll << 31) - 1);    // 4 tasks (one per warp) per CTA
  for (long long t0 = 0; t0 < n; t0 += maxg) {
    const long long nt = std::min(maxg, n - t0);
    k_eri_sq<T, LI, LJ, LK, LL><<<(unsigned)((nt + 3) / 4), 128, 0, st>>>(
        tasks + t0, nt, P.mols, P.pinfo, pp, P.cls_list, b2_boys_table<T>(P), out);
    b2_count_launches(1);
  }
}

// batch plans: the float32 classes with at most 27 components take the flattened kernel
template <typename T, int LI, int LJ, int LK, int LL>
static void b2_eri_group_batch(const B2PlanDev &P, const B2EriTask *tasks, long long n,
                               const B2PairPrim<T> *pp, T *out, cudaStream_t st) {
  constexpr int NC = (LI ? 3 : 1) * (LJ ? 3 : 1) * (LK ? 3 : 1) * (LL ? 3 : 1);
  if constexpr (std::is_same<T, float>::value && NC <= 27) {
    const long long maxg = 4 * ((1ll << 31) - 1);
    for (long long t0 = 0; t0 < n; t0 += maxg) {
      const long long nt = std::min(maxg, n - t0);
      k_eri_fl<LI, LJ, LK, LL><<<(unsigned)((nt + 3) / 4), 128, 0, st>>>(
          tasks + t0, nt, P.mols, P.pinfo, pp, P.pp32_n, P.cls_list, P.boys32, out);
      b2_count_launches(1);
    }
  } else {
    b2_eri_group<T, LI, LJ, LK, LL>(P, tasks, n, pp, out, st);
  }
}

// The 16 class kernels write disjoint entries of the s8 lists, so they run side by side: each on
// one of the plan's bucket streams (round robin, forked from and joined back to `st` with
// events), which fills the GPU across the tails of the individual launches.
template <typename T>
static void b2_eri_all(const B2PlanDev &P, const B2EriTask *tasks, const std::vector<long long> &g,
                       const B2PairPrim<T> *pp, T *out, cudaStream_t st) {
  const bool fork = P.bkt_stream[0] != nullptr;
  if (fork) cudaEventRecord(P.bkt_ev[B2_NBKT], st);
  int k = 0;
  auto sk = [&]() -> cudaStream_t {
    if (!fork) return st;
    cudaStream_t s = P.bkt_stream[k % B2_NBKT];
    if (k < B2_NBKT) cudaStreamWaitEvent(s, P.bkt_ev[B2_NBKT], 0);
    ++k;
    return s;
  };
#define B2_G(grp, LI, LJ, LK, LL)                                                            \
  if (g[grp + 1] > g[grp])                                                                   \
    b2_eri_group_batch<T, LI, LJ, LK, LL>(P, tasks + g[grp], g[grp + 1] - g[grp], pp, out, sk());
  B2_G(0, 0, 0, 0, 0) B2_G(1, 0, 0, 1, 0) B2_G(2, 0, 0, 0, 1) B2_G(3, 0, 0, 1, 1)
  B2_G(4, 1, 0, 0, 0) B2_G(5, 1, 0, 1, 0) B2_G(6, 1, 0, 0, 1) B2_G(7, 1, 0, 1, 1)
  B2_G(8, 0, 1, 0, 0) B2_G(9, 0, 1, 1, 0) B2_G(10, 0, 1, 0, 1) B2_G(11, 0, 1, 1, 1)
  B2_G(12, 1, 1, 0, 0) B2_G(13, 1, 1, 1, 0) B2_G(14, 1, 1, 0, 1) B2_G(15, 1, 1, 1, 1)
#undef B2_G
  if (fork)
    for (int b = 0; b < B2_NBKT && b < k; ++b) {
      cudaEventRecord(P.bkt_ev[b], P.bkt_stream[b]);
      cudaStreamWaitEvent(st, P.bkt_ev[b], 0);
    }
}

// Work list on the device.  Item it = 4 sp + c (sp: global bra shell pair, c: ket class) owns
// ceil(cnt / chunk) x nsub tasks, cnt = class-c kets KL <= (I,I); tasks are grouped by
// (bra class, c) and within a group ordered by item (the order of b2_eri_tasks).  Three passes
// over tiles of B2_TT items: per-tile group sums, an exclusive scan of each group over the
// tiles (group totals to the host, which sizes the list), then each tile writes its tasks.
// A 4096-molecule batch has ~6e6 items and ~1.7e7 tasks.
#define B2_TT 1024                 // items per tile: 256 threads x 4 consecutive items

__device__ __forceinline__ void b2_task_item(const B2MolDev *__restrict__ mols, int nmol,
                                             const B2PairInfo *__restrict__ pinfo,
                                             const int *__restrict__ cls_cnt, long long it, long long n_items,
                                             int chunk, int split_p, int &grp, int &n, int &mol, int &IJ,
                                             int &cnt, int &nsub) {
  grp = 0; n = 0; mol = 0; IJ = 0; cnt = 0; nsub = 1;
  if (it >= n_items) return;
  const long long sp = it >> 2;
  const int c = (int)(it & 3);
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (mols[mid].sp_off <= sp) lo = mid; else hi = mid - 1;
  }
  const B2MolDev &md = mols[lo];
  const B2PairInfo pi = pinfo[sp];
  const int spcut = (int)b2_tri(pi.I) + pi.I;
  mol = lo;
  IJ = (int)(sp - md.sp_off);
  cnt = cls_cnt[4ll * md.sp_off + (long long)c * md.nsp + spcut];
  nsub = (split_p && pi.lI) ? 3 : 1;
  grp = (pi.lI + 2 * pi.lJ) * 4 + c;
  n = (cnt + chunk - 1) / chunk * nsub;
}

__global__ void __launch_bounds__(256)
k_task_tile_sums(const B2MolDev *__restrict__ mols, int nmol, const B2PairInfo *__restrict__ pinfo,
                 const int *__restrict__ cls_cnt, long long n_items, int chunk, int split_p,
                 long long *__restrict__ tile_sum) {
  __shared__ int s[16];
  if (threadIdx.x < 16) s[threadIdx.x] = 0;
  __syncthreads();
  const long long i0 = (long long)blockIdx.x * B2_TT + 4 * threadIdx.x;
  for (int k = 0; k < 4; ++k) {
    int grp, n, mol, IJ, cnt, nsub;
    b2_task_item(mols, nmol, pinfo, cls_cnt, i0 + k, n_items, chunk, split_p, grp, n, mol, IJ, cnt, nsub);
    if (n) atomicAdd(&s[grp], n);
  }
  __syncthreads();
  if (threadIdx.x < 16) tile_sum[(long long)blockIdx.x * 16 + threadIdx.x] = s[threadIdx.x];
}

// one CTA per group: exclusive scan of the group's tile sums in place; total -> gtot[group]
__global__ void __launch_bounds__(1024)
k_task_scan(long long *__restrict__ tile_sum, long long ntile, long long *__restrict__ gtot) {
  __shared__ long long wsum[32];
  const int g = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long carry = 0;
  for (long long t0 = 0; t0 < ntile; t0 += 1024) {
    const long long t = t0 + threadIdx.x;
    const long long v = t < ntile ? tile_sum[t * 16 + g] : 0;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      long long z = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= o) z += y;
      }
      wsum[lane] = z;                                    // inclusive over warps
    }
    __syncthreads();
    const long long excl = carry + (w ? wsum[w - 1] : 0) + x - v;
    if (t < ntile) tile_sum[t * 16 + g] = excl;
    carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) gtot[g] = carry;
}

__global__ void __launch_bounds__(256)
k_task_write(const B2MolDev *__restrict__ mols, int nmol, const B2PairInfo *__restrict__ pinfo,
             const int *__restrict__ cls_cnt, long long n_items, int chunk, int split_p,
             const long long *__restrict__ tile_base, const long long *__restrict__ goff,
             B2EriTask *__restrict__ tasks) {
  __shared__ long long wsum[8][16];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long i0 = (long long)blockIdx.x * B2_TT + 4 * threadIdx.x;
  int grp[4], n[4], mol[4], IJ[4], cnt[4], nsub[4];
  for (int k = 0; k < 4; ++k)
    b2_task_item(mols, nmol, pinfo, cls_cnt, i0 + k, n_items, chunk, split_p, grp[k], n[k], mol[k], IJ[k],
                 cnt[k], nsub[k]);
  // per group: exclusive prefix of this thread's task counts over the CTA (warp scans + warp sums)
  long long off[4];
  for (int g = 0; g < 16; ++g) {
    int v = 0;
    for (int k = 0; k < 4; ++k) v += grp[k] == g ? n[k] : 0;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w][g] = x;
    int run = x - v;                                     // exclusive within the warp
    for (int k = 0; k < 4; ++k)
      if (grp[k] == g) { off[k] = run; run += n[k]; }
  }
  __syncthreads();
  for (int k = 0; k < 4; ++k) {
    if (!n[k]) continue;
    const int g = grp[k];
    long long o = goff[g] + tile_base[(long long)blockIdx.x * 16 + g] + off[k];
    for (int v = 0; v < w; ++v) o += wsum[v][g];
    const int c = (int)((i0 + k) & 3);
    for (int s0 = 0; s0 < cnt[k]; s0 += chunk)
      for (int sub = 0; sub < nsub[k]; ++sub)
        tasks[o++] = B2EriTask{mol[k], IJ[k], c, s0, min(chunk, cnt[k] - s0), nsub[k] > 1 ? sub : -1};
  }
}

static int b2_eri_task_upload(B2PlanDev &P, int precision, cudaStream_t st) {
  B2EriTask *&dst = precision == 64 ? P.eri_tasks64 : P.eri_tasks32;
  std::vector<long long> &goff = precision == 64 ? P.eri_goff64 : P.eri_goff32;
  if (dst) return B2_OK;
  const int chunk = 32;                          // kets per warp task
  const int split_p = precision == 64 ? 1 : 0;
  const long long n_items = 4ll * P.h.n_sp;
  const long long ntile = std::max(1ll, (n_items + B2_TT - 1) / B2_TT);
  long long *scratch = nullptr;                  // tile sums (16 per tile), group totals, group starts
  B2_CUDA_TRY(b2_dmalloc_t(&scratch, sizeof(long long) * (size_t)(16 * ntile + 32), st));
  long long *gtot = scratch + 16 * ntile, *dgoff = gtot + 16;
  std::vector<long long> tot(16, 0);
  int rc = B2_OK;
  if (n_items > 0) {
    k_task_tile_sums<<<(unsigned)ntile, 256, 0, st>>>(P.mols, P.h.nmol, P.pinfo, P.cls_cnt, n_items, chunk,
                                                      split_p, scratch);
    k_task_scan<<<16, 1024, 0, st>>>(scratch, ntile, gtot);
    b2_count_launches(2);
    if (cudaMemcpyAsync(tot.data(), gtot, sizeof(long long) * 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rc = B2_ERR_CUDA;
  }
  std::vector<long long> g(17, 0);
  for (int k = 0; k < 16; ++k) g[k + 1] = g[k] + tot[k];
  if (!rc && g[16] >= (1ll << 31)) rc = B2_ERR_SIZE;
  if (!rc && b2_dmalloc_t(&dst, sizeof(B2EriTask) * std::max<size_t>(1, (size_t)g[16]), st) != cudaSuccess) {
    dst = nullptr;
    rc = B2_ERR_CUDA;
  }
  if (!rc && n_items > 0) {
    if (cudaMemcpyAsync(dgoff, g.data(), sizeof(long long) * 16, cudaMemcpyHostToDevice, st) != cudaSuccess)
      rc = B2_ERR_CUDA;
    else {
      k_task_write<<<(unsigned)ntile, 256, 0, st>>>(P.mols, P.h.nmol, P.pinfo, P.cls_cnt, n_items, chunk,
                                                    split_p, scratch, dgoff, dst);
      b2_count_launches(1);
      if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) rc = B2_ERR_CUDA;
    }
  }
  b2_dfree(scratch, st);
  if (rc) {
    b2_dfree(dst, st);
    dst = nullptr;
    return rc;
  }
  goff = g;
  return B2_OK;
}

int b2_eri_tasks_ready(B2PlanDev &P, int precision, cudaStream_t st) {
  if (precision != 64 && precision != 32) return B2_ERR_ARG;
  return b2_eri_task_upload(P, precision, st);
}

int b2_launch_eri_s8(B2PlanDev &P, int precision, void *out, cudaStream_t st) {
  if (precision != 64 && precision != 32) return B2_ERR_ARG;
  int rc = b2_eri_task_upload(P, precision, st);
  if (rc) return rc;
  if (precision == 64)
    b2_eri_all<double>(P, P.eri_tasks64, P.eri_goff64, P.pp64, (double *)out, st);
  else
    b2_eri_all<float>(P, P.eri_tasks32, P.eri_goff32, P.pp32, (float *)out, st);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

// ============================================================================================
// Allocation-free single-molecule ERI entry (b2_int2e_sph_s8_noalloc).
//
// For callers that must not call cudaMalloc: processes whose device memory is handed out by
// another allocator or a pool with a fixed budget (a cudaMalloc there would fail or take memory
// the pool has promised elsewhere), and loops with a latency budget, where cudaMalloc/cudaFree
// can block and synchronise the device.  The per-molecule tables the ERI kernels read (molecule
// descriptor, shell-pair primitive data, class lists, work list, Boys table) live in one
// file-scope __device__ array of B2_NOALLOC_BYTES (2.5 MiB) that every GPU loading this library
// keeps until the process exits; the host side fills a static buffer of the same size and copies
// it with one cudaMemcpyAsync (pageable source: the copy has left the buffer when the call
// returns).  Limits: nbas <= 48 shells, nao <= 70, s/p shells with <= 3 primitives.  The s8
// output is written completely, so no part of the array has to start at zero.
// The call is asynchronous on `stream`: the output is ready, and kernel faults are reported,
// only once the caller synchronises that stream.  All calls share the device array and the
// host staging buffer: calls from several host threads must be serialised by the caller, and
// calls whose work overlaps on the GPU (different streams) race; calls on one stream are
// ordered.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make it before any stream capture.
#define B2_NOALLOC_MAXBAS 48
#define B2_NOALLOC_MAXSP (B2_NOALLOC_MAXBAS * (B2_NOALLOC_MAXBAS + 1) / 2)
#define B2_NOALLOC_MAXTASK (B2_NOALLOC_MAXSP * 42)
#define B2_NOALLOC_BYTES (2621440)

static __device__ __align__(256) unsigned char g_b2_noalloc_scratch[B2_NOALLOC_BYTES];
static __align__(256) unsigned char g_b2_noalloc_stage[B2_NOALLOC_BYTES];
static unsigned char *g_b2_noalloc_dev[128];     // device address of the array, per device

static size_t b2_na_align(size_t x) { return (x + 255) & ~(size_t)255; }

// class-group launch over a fixed-size group table (no container)
template <typename T>
static void b2_eri_all_na(const B2PlanDev &P, const B2EriTask *tasks, const long long *g,
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

extern "C" int b2_int2e_sph_s8_noalloc(const int *atm, int natm, const int *bas, int nbas,
                                       const double *env, int n_env, int precision, void *eri_out,
                                       void *stream) {
  if (!atm || !bas || !env || !eri_out || natm <= 0 || nbas <= 0 || n_env <= 0) return B2_ERR_ARG;
  if (precision != 64 && precision != 32) return B2_ERR_ARG;
  if (nbas > B2_NOALLOC_MAXBAS) return B2_ERR_SIZE;
  unsigned char *H = g_b2_noalloc_stage;
  // ---- host tables in the static staging buffer (same layout as the device array) ----
  const size_t o_mol = 0;
  const size_t o_pi = b2_na_align(o_mol + sizeof(B2MolDev));
  const size_t o_pp = b2_na_align(o_pi + sizeof(B2PairInfo) * B2_NOALLOC_MAXSP);
  const size_t pp_bytes = (precision == 64 ? sizeof(B2PairPrim<double>) : sizeof(B2PairPrim<float>)) *
                          B2_NOALLOC_MAXSP * B2_MAXPP;
  const size_t o_cls = b2_na_align(o_pp + pp_bytes);
  const size_t o_task = b2_na_align(o_cls + sizeof(int) * B2_NOALLOC_MAXSP);
  const size_t o_boys = b2_na_align(o_task + sizeof(B2EriTask) * B2_NOALLOC_MAXTASK);
  const size_t total = b2_na_align(o_boys + sizeof(double) * B2_BOYS_NT * B2_BOYS_NM);
  if (total > B2_NOALLOC_BYTES) return B2_ERR_SIZE;
  B2Shell S[B2_NOALLOC_MAXBAS];
  int nao = 0;
  for (int s = 0; s < nbas; ++s) {
    const int *b = bas + s * B2_BAS_SLOTS;
    const int l = b[B2_ANG_OF], np = b[B2_NPRIM_OF], ia = b[B2_ATOM_OF];
    if (l > B2_MAXL || np < 1 || np > B2_MAXPRIM || b[B2_NCTR_OF] != 1) return B2_ERR_UNSUPPORTED;
    if (ia < 0 || ia >= natm) return B2_ERR_ARG;
    const int pc = atm[ia * B2_ATM_SLOTS + B2_PTR_COORD];
    if (pc < 0 || pc + 3 > n_env || b[B2_PTR_EXP] < 0 || b[B2_PTR_COEFF] < 0 ||
        b[B2_PTR_EXP] + np > n_env || b[B2_PTR_COEFF] + np > n_env)
      return B2_ERR_ARG;
    memset(&S[s], 0, sizeof(B2Shell));
    for (int d = 0; d < 3; ++d) S[s].R[d] = env[pc + d];
    const double fac = l == 0 ? B2_FAC_S : B2_FAC_P;
    for (int k = 0; k < np; ++k) {
      S[s].exp[k] = env[b[B2_PTR_EXP] + k];
      S[s].coef[k] = env[b[B2_PTR_COEFF] + k] * fac;
    }
    S[s].l = l; S[s].ao0 = nao; S[s].nprim = np; S[s].atom = ia;
    nao += 2 * l + 1;
  }
  if (nao > B2_MAXNAO - 2) return B2_ERR_SIZE;
  const int nsp = nbas * (nbas + 1) / 2;
  B2MolDev *md = (B2MolDev *)(H + o_mol);
  memset(md, 0, sizeof(B2MolDev));
  md->nao = nao; md->nbas = nbas; md->natm = natm; md->nsp = nsp;
  const long long n2 = (long long)nao * (nao + 1) / 2;
  md->n4 = n2 * (n2 + 1) / 2;
  B2PairInfo *PI = (B2PairInfo *)(H + o_pi);
  static int cls[B2_NOALLOC_MAXSP];
  for (int I = 0; I < nbas; ++I)
    for (int J = 0; J <= I; ++J) {
      const int sp = (int)b2_tri(I) + J;
      const B2Shell &a = S[I], &b = S[J];
      PI[sp] = B2PairInfo{I, J, a.l, b.l, a.ao0, b.ao0, a.nprim * b.nprim, 0};
      cls[sp] = a.l + 2 * b.l;
      B2PairPrim<double> q64[B2_MAXPP];
      B2PairPrim<float> q32[B2_MAXPP];
      b2_pair_prims_packed(a, b, q64, q32);              // same screening as the batch plan
      for (int x = 0; x < B2_MAXPP; ++x) {
        if (precision == 64) ((B2PairPrim<double> *)(H + o_pp))[(size_t)sp * B2_MAXPP + x] = q64[x];
        else ((B2PairPrim<float> *)(H + o_pp))[(size_t)sp * B2_MAXPP + x] = q32[x];
      }
    }
  int *CL = (int *)(H + o_cls);
  int start = 0;
  for (int c = 0; c < 4; ++c) {
    md->cls_start[c] = start;
    for (int sp = 0; sp < nsp; ++sp)
      if (cls[sp] == c) CL[start++] = sp;
  }
  md->cls_start[4] = start;
  // work list grouped by class combination, kets in chunks of 128 (as b2_eri_tasks)
  B2EriTask *TK = (B2EriTask *)(H + o_task);
  long long goff[17];
  long long nt = 0;
  for (int grp = 0; grp < 16; ++grp) {
    goff[grp] = nt;
    const int bc = grp / 4, c = grp % 4;
    for (int IJ = 0; IJ < nsp; ++IJ) {
      if (PI[IJ].lI + 2 * PI[IJ].lJ != bc) continue;
      const int spcut = (int)b2_tri(PI[IJ].I) + PI[IJ].I;
      int cnt = 0;                                      // class-c members KL <= spcut
      for (int e = md->cls_start[c]; e < md->cls_start[c + 1]; ++e) cnt += (CL[e] <= spcut);
      const int nsub = (precision == 64 && PI[IJ].lI) ? 3 : 1;
      for (int s0 = 0; s0 < cnt; s0 += 128)
        for (int sub = 0; sub < nsub; ++sub) {
          if (nt >= B2_NOALLOC_MAXTASK) return B2_ERR_SIZE;
          TK[nt++] = B2EriTask{0, IJ, c, s0, cnt - s0 < 128 ? cnt - s0 : 128, nsub > 1 ? sub : -1};
        }
    }
  }
  goff[16] = nt;
  b2_boys_fill_table((double *)(H + o_boys));
  if (precision == 32) {                          // float32 kernels read a float table
    const double *bd = (const double *)(H + o_boys);
    float *bf = (float *)(H + o_boys);
    for (int i = 0; i < B2_BOYS_NT * B2_BOYS_NM; ++i) bf[i] = (float)bd[i];   // in place, ascending
  }
  // ---- stage to the device array and launch (no device allocation anywhere) ----
  // arguments are all checked above, before any CUDA call; first call on a device: set-up
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return B2_ERR_CUDA;
  if (!g_b2_noalloc_dev[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_b2_noalloc_scratch) != cudaSuccess || !p) return B2_ERR_CUDA;
    g_b2_noalloc_dev[dev] = (unsigned char *)p;
  }
  unsigned char *Dv = g_b2_noalloc_dev[dev];
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(Dv, H, total, cudaMemcpyHostToDevice, st) != cudaSuccess) return B2_ERR_CUDA;
  B2PlanDev P;                                           // view onto the static array
  P.mols = (B2MolDev *)(Dv + o_mol);
  P.pinfo = (B2PairInfo *)(Dv + o_pi);
  P.cls_list = (int *)(Dv + o_cls);
  P.boys = (double *)(Dv + o_boys);
  P.boys32 = (float *)(Dv + o_boys);
  B2EriTask *tasks = (B2EriTask *)(Dv + o_task);
  if (precision == 64)
    b2_eri_all_na<double>(P, tasks, goff, (const B2PairPrim<double> *)(Dv + o_pp), (double *)eri_out, st);
  else
    b2_eri_all_na<float>(P, tasks, goff, (const B2PairPrim<float> *)(Dv + o_pp), (float *)eri_out, st);
  P.mols = nullptr; P.pinfo = nullptr; P.cls_list = nullptr; P.boys = nullptr; P.boys32 = nullptr;
  if (cudaGetLastError() != cudaSuccess) return B2_ERR_CUDA;
  return B2_OK;
}

// primitive-pair tables of every shell pair of the batch (float64 and float32 copies, screened
// and packed), one thread per shell pair; same code as the host test build
__global__ void k_pair_prims(const B2MolDev *__restrict__ mols, int nmol, const B2Shell *__restrict__ shells,
                             const B2PairInfo *__restrict__ pinfo, long long n_sp,
                             B2PairPrim<double> *__restrict__ pp64, B2PairPrim<float> *__restrict__ pp32,
                             unsigned char *__restrict__ pp32_n) {
  const long long gp = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gp >= n_sp) return;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (mols[mid].sp_off <= gp) lo = mid; else hi = mid - 1;
  }
  const B2PairInfo pi = pinfo[gp];
  const int sh = mols[lo].sh_off;
  int n32 = 0;
  b2_pair_prims_packed(shells[sh + pi.I], shells[sh + pi.J], pp64 + gp * B2_MAXPP, pp32 + gp * B2_MAXPP, &n32);
  pp32_n[gp] = (unsigned char)n32;
}

// shell-pair tables of every molecule, one warp per molecule: pair info, the class lists
// (pairs of each angular class in ascending order, from cls_start) and the inclusive class
// prefix counts cls_cnt[4 sp_off + c nsp + sp] = #{class-c pairs <= sp}; the host test build
// fills the same tables (b2_plan_build with pair tables)
__global__ void __launch_bounds__(256)
k_plan_pairs(const B2MolDev *__restrict__ mols, int nmol, const B2Shell *__restrict__ shells,
             B2PairInfo *__restrict__ pinfo, int *__restrict__ cls_list, int *__restrict__ cls_cnt) {
  const int m = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (m >= nmol) return;                           // whole warp
  const B2MolDev md = mols[m];
  const B2Shell *S = shells + md.sh_off;
  const unsigned le = (2u << lane) - 1u;           // lanes <= this one (lane 31: all)
  int run[4] = {0, 0, 0, 0};
  for (int base = 0; base < md.nsp; base += 32) {
    const int sp = base + lane;
    int c = -1;
    if (sp < md.nsp) {
      const int I = (int)b2_untri(sp), J = sp - (int)b2_tri(I);
      const int lI = S[I].l, lJ = S[J].l;
      pinfo[md.sp_off + sp] = B2PairInfo{I, J, lI, lJ, S[I].ao0, S[J].ao0, S[I].nprim * S[J].nprim, 0};
      c = b2_class(lI, lJ);
    }
    for (int cc = 0; cc < 4; ++cc) {
      const unsigned mk = __ballot_sync(0xffffffffu, c == cc);
      const int incl = run[cc] + __popc(mk & le);
      if (sp < md.nsp) cls_cnt[4ll * md.sp_off + (long long)cc * md.nsp + sp] = incl;
      if (c == cc) cls_list[md.sp_off + md.cls_start[cc] + incl - 1] = sp;
      run[cc] += __popc(mk);
    }
  }
}

int b2_build_pairs(B2PlanDev &P, cudaStream_t st) {
  const long long nsp = P.h.n_sp, n = nsp * B2_MAXPP;
  B2_CUDA_TRY(b2_dmalloc_t(&P.pinfo, sizeof(B2PairInfo) * (size_t)std::max(1ll, nsp), st));
  B2_CUDA_TRY(b2_dmalloc_t(&P.cls_list, sizeof(int) * (size_t)std::max(1ll, nsp), st));
  B2_CUDA_TRY(b2_dmalloc_t(&P.cls_cnt, sizeof(int) * (size_t)std::max(1ll, 4 * nsp), st));
  B2_CUDA_TRY(b2_dmalloc_t(&P.pp64, sizeof(B2PairPrim<double>) * (size_t)std::max(1ll, n), st));
  B2_CUDA_TRY(b2_dmalloc_t(&P.pp32, sizeof(B2PairPrim<float>) * (size_t)std::max(1ll, n), st));
  B2_CUDA_TRY(b2_dmalloc_t(&P.pp32_n, (size_t)std::max(1ll, nsp), st));
  if (n > 0) {
    k_plan_pairs<<<(unsigned)((P.h.nmol + 7) / 8), 256, 0, st>>>(P.mols, P.h.nmol, P.shells, P.pinfo,
                                                                 P.cls_list, P.cls_cnt);
    k_pair_prims<<<(unsigned)((nsp + 127) / 128), 128, 0, st>>>(P.mols, P.h.nmol, P.shells, P.pinfo,
                                                               nsp, P.pp64, P.pp32, P.pp32_n);
    b2_count_launches(2);
    B2_CUDA_TRY(cudaGetLastError());
  }
  return B2_OK;
}

// Work the float32 ERI kernels do for a plan: primitive quartets evaluated (bra survivors x ket
// survivors of every shell quartet of the task list) and their arithmetic by the per-class
// counts of eri_flops.h (generated from eri_sq.cuh by eri_flops_count.cu).  One thread per task.
__global__ void __launch_bounds__(256)
k_eri_count(const B2EriTask *__restrict__ tasks, long long n, const B2MolDev *__restrict__ mols,
            const int *__restrict__ cls_list, const unsigned char *__restrict__ ppn, double fl, double sp,
            double *__restrict__ out) {
  __shared__ double red[3][8];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double q = 0;
  if (t < n) {
    const B2EriTask tk = tasks[t];
    const B2MolDev md = mols[tk.mol];
    const double nb = ppn[md.sp_off + tk.IJ];
    int nq = 0;
    for (int k = 0; k < tk.count; ++k) nq += ppn[md.sp_off + cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + k]];
    q = nb * nq;
  }
  double v[3] = {q, q * fl, q * sp};
  for (int c = 0; c < 3; ++c)
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 3; ++c) red[c][threadIdx.x >> 5] = v[c];
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0;
    for (int w = 0; w < 8; ++w) s += red[threadIdx.x][w];
    atomicAdd(&out[threadIdx.x], s);
  }
}

int b2_launch_eri_count(B2PlanDev &P, double *host_out) {
  int rc = b2_eri_task_upload(P, 32, nullptr);
  if (rc) return rc;
  double *d = nullptr;
  B2_CUDA_TRY(b2_dmalloc_t(&d, 3 * sizeof(double)));
  B2_CUDA_TRY(cudaMemset(d, 0, 3 * sizeof(double)));
  const std::vector<long long> &g = P.eri_goff32;
  for (int grp = 0; grp < 16; ++grp) {
    const long long n = g[grp + 1] - g[grp];
    if (n <= 0) continue;
    k_eri_count<<<(unsigned)((n + 255) / 256), 256>>>(P.eri_tasks32 + g[grp], n, P.mols, P.cls_list, P.pp32_n,
                                                       (double)B2_ERI_FLOPS[grp], (double)B2_ERI_SPECIAL[grp], d);
    b2_count_launches(1);
  }
  rc = cudaMemcpy(host_out, d, 3 * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess ? B2_OK : B2_ERR_CUDA;
  b2_dfree(d);
  return rc;
}
