// extern "C" entry points of libb200dft.so (declared in include/b200dft.h).
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include "device_plan.cuh"
#include "devmem.cuh"
#include "xc.cuh"
#include "scf.cuh"
#include "xc_math.cuh"
#include "setup.cuh"
#include "b200dft.h"             // after the enum of status codes in common.cuh (same values)

static thread_local std::string g_last_error;
#include <atomic>
#include <mutex>
static std::atomic<long long> g_b2_launches{0};
void b2_count_launches(long long n) { g_b2_launches += n; }

static int b2_note(cudaError_t e) {
  if (e != cudaSuccess) { g_last_error = cudaGetErrorString(e); return B2_ERR_CUDA; }
  return B2_OK;
}

#define B2_TRY(x) do { int _rc = b2_note(x); if (_rc) return _rc; } while (0)

static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64] = {};

static cudaError_t b2_pool(cudaMemPool_t *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    uint64_t keep = ~0ull;
    int no = 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

cudaError_t b2_dmalloc(void **p, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool = nullptr;
  cudaError_t e = b2_pool(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st);
}

void b2_dfree(void *p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

// Plan uploads: every table is packed into one pinned staging buffer (kept and reused by later
// plans, grown when a larger batch needs it) and copied with cudaMemcpyAsync on the plan's
// stream; the staging lock is held until that stream has been synchronized.
struct B2Upload {
  cudaStream_t st = nullptr;
  unsigned char *stage = nullptr;
  size_t cap = 0, used = 0, bytes = 0;
};
static std::mutex g_stage_mu;
static unsigned char *g_stage = nullptr;
static size_t g_stage_cap = 0;

// device copy of a host table: staged and queued with an upload context, else synchronous
template <typename T>
static int b2_upload(T **dst, const std::vector<T> &src, B2Upload *u = nullptr) {
  size_t n = std::max<size_t>(1, src.size());
  B2_TRY(b2_dmalloc_t(dst, sizeof(T) * n, u ? u->st : nullptr));
  if (src.empty()) return B2_OK;
  const size_t nb = sizeof(T) * src.size();
  if (!u) {
    B2_TRY(cudaMemcpy(*dst, src.data(), nb, cudaMemcpyHostToDevice));
    return B2_OK;
  }
  const size_t at = (u->used + 255) / 256 * 256;
  if (at + nb > u->cap) return B2_ERR_SIZE;
  std::memcpy(u->stage + at, src.data(), nb);
  B2_TRY(cudaMemcpyAsync(*dst, u->stage + at, nb, cudaMemcpyHostToDevice, u->st));
  u->used = at + nb;
  u->bytes += nb;
  return B2_OK;
}

static void b2_subset_free(B2PlanDev *P) {
  b2_dfree(P->sub.mol_map); b2_dfree(P->sub.jk_off); b2_dfree(P->sub.x32); b2_dfree(P->sub.x64);
  b2_dfree(P->sub.xtc); b2_dfree(P->sub.sv_off); b2_dfree(P->sub.bkt_map);
  b2_dfree(P->sub.xq_items);
  P->sub = B2SubsetDev();
}

// frees go to the legacy stream (after all work queued on blocking streams); the plan's own
// bucket streams are drained first
static void b2_plan_free(B2PlanDev *P) {
  if (!P) return;
  for (int b = 0; b < B2_NBKT; ++b) if (P->bkt_stream[b]) cudaStreamSynchronize(P->bkt_stream[b]);
  if (P->jk_stream) cudaStreamSynchronize(P->jk_stream);
  b2_subset_free(P);
  b2_grid_free(*P);
  b2_dfree(P->mols); b2_dfree(P->row_off); b2_dfree(P->shells); b2_dfree(P->pinfo);
  b2_dfree(P->pp64); b2_dfree(P->pp32); b2_dfree(P->pp32_n); b2_dfree(P->ao2sh); b2_dfree(P->cls_list);
  b2_dfree(P->cls_cnt); b2_dfree(P->atom_xyz); b2_dfree(P->atom_z); b2_dfree(P->boys); b2_dfree(P->boys32);
  b2_dfree(P->jk_chunk_off);
  b2_dfree(P->eri_tasks32); b2_dfree(P->eri_tasks64);
  b2_dfree(P->sv_off); b2_dfree(P->sv_work); b2_dfree(P->bkt_map);
  for (int b = 0; b < B2_NBKT; ++b) if (P->bkt_stream[b]) cudaStreamDestroy(P->bkt_stream[b]);
  for (int b = 0; b <= B2_NBKT; ++b) if (P->bkt_ev[b]) cudaEventDestroy(P->bkt_ev[b]);
  if (P->jk_stream) cudaStreamDestroy(P->jk_stream);
  for (int k = 0; k < 2; ++k) if (P->jk_ev[k]) cudaEventDestroy(P->jk_ev[k]);
  delete P;
}

static int b2_set_jk_chunk(B2PlanDev *P, long long elems, B2Upload *u = nullptr) {
  // whole runs of 8 for every thread of a 1024-thread CTA; at most 32768 entries per CTA
  // keeps the fixed-point J/K accumulators exact
  if (elems <= 0) elems = 32768;
  elems = std::min(32768LL, (elems + 8191) / 8192 * 8192);
  const int nmol = P->h.nmol;
  std::vector<long long> off(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) off[m + 1] = off[m] + (P->h.mols[m].n4 + elems - 1) / elems;
  b2_dfree(P->jk_chunk_off);
  P->jk_chunk_off = nullptr;
  P->jk_off_h = std::move(off);
  int rc = b2_upload(&P->jk_chunk_off, P->jk_off_h, u);
  if (rc) return rc;
  P->jk_chunk = elems;
  P->jk_nchunks = P->jk_off_h[nmol];
  return B2_OK;
}

// molecules (a list of indices) grouped by orbital bucket, order kept within a bucket
static void b2_buckets(const B2PlanDev *P, const std::vector<int> &mols, std::vector<int> &map,
                       std::vector<int> &off) {
  off.assign(B2_NBKT + 1, 0);
  auto bkt = [&](int m) { return std::min(B2_NBKT - 1, (P->h.mols[m].nao - 1) / 16); };
  for (int m : mols) ++off[bkt(m) + 1];
  for (int b = 0; b < B2_NBKT; ++b) off[b + 1] += off[b];
  map.assign(mols.size(), 0);
  std::vector<int> pos(off.begin(), off.end() - 1);
  for (int m : mols) map[pos[bkt(m)]++] = m;
}

// warp-task table of the J/K products and their pair-vector workspace
static int b2_set_sv(B2PlanDev *P, B2Upload *u) {
  const int nmol = P->h.nmol;
  std::vector<long long> off(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    const long long N = P->h.mols[m].nao;
    off[m + 1] = off[m] + b2_sv_tasks_host(N * (N + 1) / 2);
  }
  P->sv_off_h = off;
  int rc = b2_upload(&P->sv_off, P->sv_off_h, u);
  if (rc) return rc;
  P->sv_ntask = off[nmol];
  B2_TRY(b2_dmalloc_t(&P->sv_work, sizeof(double) * 4 * (size_t)std::max(1ll, P->h.n_rows), u ? u->st : nullptr));
  std::vector<int> all(nmol);
  for (int m = 0; m < nmol; ++m) all[m] = m;
  b2_buckets(P, all, P->bkt_map_h, P->bkt_off_h);
  for (int b = 0; b < B2_NBKT; ++b) B2_TRY(cudaStreamCreateWithFlags(&P->bkt_stream[b], cudaStreamNonBlocking));
  for (int b = 0; b <= B2_NBKT; ++b) B2_TRY(cudaEventCreateWithFlags(&P->bkt_ev[b], cudaEventDisableTiming));
  B2_TRY(cudaStreamCreateWithFlags(&P->jk_stream, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k) B2_TRY(cudaEventCreateWithFlags(&P->jk_ev[k], cudaEventDisableTiming));
  return b2_upload(&P->bkt_map, P->bkt_map_h, u);
}

extern "C" {

int b2_version(void) { return 100; }

int b2_launch_count(int64_t *out) {
  if (!out) return B2_ERR_ARG;
  *out = g_b2_launches.load();
  return B2_OK;
}

const char *b2_last_error(void) { return g_last_error.c_str(); }

int b2_plan_create(int nmol, const int *natm, const int *nbas, const int *atm, const int *bas,
                   const double *env, const int64_t *env_off, void **plan) {
  if (nmol <= 0 || !natm || !nbas || !atm || !bas || !env || !env_off || !plan) return B2_ERR_ARG;
  B2PlanDev *P = new B2PlanDev();
  int rc = b2_plan_build(P->h, nmol, natm, nbas, atm, bas, env, (const long long *)env_off,
                         /*pair_tables=*/false);
  if (rc) { delete P; return rc; }
  // every upload and table kernel goes to one non-blocking stream, synchronized once at the end
  // (no ordering with, or wait on, work the caller has queued elsewhere on the device)
  std::vector<double> tab(B2_BOYS_NT * B2_BOYS_NM);
  b2_boys_fill_table(tab.data());
  std::vector<float> tab32(tab.begin(), tab.end());
  const B2PlanHost &H = P->h;
  size_t need = 16 * 256 + sizeof(B2MolDev) * H.mols.size() + sizeof(long long) * H.row_off.size() +
                sizeof(B2Shell) * H.shells.size() + sizeof(int) * H.ao2sh.size() +
                sizeof(double) * H.atom_xyz.size() + sizeof(int) * H.atom_z.size() +
                sizeof(double) * tab.size() + sizeof(float) * tab32.size() +
                (2 * sizeof(long long) + sizeof(int)) * (size_t)(nmol + 1);
  std::lock_guard<std::mutex> lock(g_stage_mu);
  if (need > g_stage_cap) {
    if (g_stage) cudaFreeHost(g_stage);
    g_stage = nullptr;
    g_stage_cap = 0;
    const size_t cap = need + need / 4;
    if ((rc = b2_note(cudaMallocHost((void **)&g_stage, cap)))) { delete P; return rc; }
    g_stage_cap = cap;
  }
  B2Upload u;
  u.stage = g_stage;
  u.cap = g_stage_cap;
  if ((rc = b2_note(cudaStreamCreateWithFlags(&u.st, cudaStreamNonBlocking)))) { delete P; return rc; }
  if ((rc = b2_upload(&P->mols, H.mols, &u)) || (rc = b2_upload(&P->row_off, H.row_off, &u)) ||
      (rc = b2_upload(&P->shells, H.shells, &u)) || (rc = b2_upload(&P->ao2sh, H.ao2sh, &u)) ||
      (rc = b2_upload(&P->atom_xyz, H.atom_xyz, &u)) || (rc = b2_upload(&P->atom_z, H.atom_z, &u)) ||
      (rc = b2_upload(&P->boys, tab, &u)) || (rc = b2_upload(&P->boys32, tab32, &u)) ||
      (rc = b2_set_jk_chunk(P, 0, &u)) || (rc = b2_build_pairs(*P, u.st)) || (rc = b2_set_sv(P, &u))) {
    cudaStreamSynchronize(u.st);
    cudaStreamDestroy(u.st);
    b2_plan_free(P);
    return rc;
  }
  rc = b2_note(cudaStreamSynchronize(u.st));
  cudaStreamDestroy(u.st);
  if (rc) { b2_plan_free(P); return rc; }
  P->h2d_bytes = (long long)u.bytes;
  cudaGetDevice(&P->device);
  *plan = P;
  return B2_OK;
}

int b2_release_cached_memory(void) {
  std::lock_guard<std::mutex> lock(g_pool_mu);
  for (int d = 0; d < 64; ++d)
    if (g_pool[d] && cudaMemPoolTrimTo(g_pool[d], 0) != cudaSuccess) return b2_note(cudaGetLastError());
  return B2_OK;
}

int b2_plan_h2d_bytes(void *plan, int64_t *bytes) {
  if (!plan || !bytes) return B2_ERR_ARG;
  *bytes = ((B2PlanDev *)plan)->h2d_bytes;
  return B2_OK;
}

int b2_plan_destroy(void *plan) {
  b2_plan_free((B2PlanDev *)plan);
  return B2_OK;
}

int b2_plan_info(void *plan, int64_t *info) {
  if (!plan || !info) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  info[0] = P->h.n_eri; info[1] = P->h.n_mat; info[2] = P->h.nmol; info[3] = P->h.max_nao;
  info[4] = P->h.n_rows; info[5] = P->h.n_sp; info[6] = P->jk_chunk; info[7] = P->jk_nchunks;
  return B2_OK;
}

int b2_plan_offsets(void *plan, int64_t *eri_off, int64_t *mat_off, int *nao, int *nocc) {
  if (!plan) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  for (int m = 0; m < P->h.nmol; ++m) {
    if (eri_off) eri_off[m] = P->h.mols[m].eri_off;
    if (mat_off) mat_off[m] = P->h.mols[m].mat_off;
    if (nao) nao[m] = P->h.mols[m].nao;
    if (nocc) nocc[m] = P->h.mols[m].nocc;
  }
  return B2_OK;
}

int b2_plan_set_jk_chunk(void *plan, int64_t elems) {
  if (!plan) return B2_ERR_ARG;
  return b2_set_jk_chunk((B2PlanDev *)plan, elems);
}

int b2_plan_set_xc_impl(void *plan, int impl) {
  if (!plan || impl < 0 || impl > 2) return B2_ERR_ARG;
  ((B2PlanDev *)plan)->xc_impl = impl;
  return B2_OK;
}

int b2_plan_set_xc_tiles(void *plan, int tiles_per_cta) {
  if (!plan || tiles_per_cta < 0) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  b2_subset_free(P);                  // subset tables derive from the tile split
  return b2_xc_set_tpc(*P, tiles_per_cta);
}

int b2_plan_set_xc_bucket_tiles(void *plan, const int *tiles) {
  if (!plan || !tiles) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  if (!P->g.grid_off) return B2_ERR_ARG;
  for (int b = 0; b < B2_NBKT; ++b)
    if (tiles[b] < 0 || tiles[b] > 1024) return B2_ERR_ARG;
  b2_subset_free(P);                  // subset tables derive from the tile split
  for (int b = 0; b < B2_NBKT; ++b) P->g.xq_tpc[b] = tiles[b];
  std::vector<int> all(P->h.nmol);
  for (int m = 0; m < P->h.nmol; ++m) all[m] = m;
  return b2_xq_build(*P, all, &P->g.xq_items, P->g.xq_off_h);
}

int b2_xc_tc_status(int reset, int *status) {
  if (!status) return B2_ERR_ARG;
  const int v = b2_xc_tc_status_read(reset);
  if (v < 0) return B2_ERR_CUDA;
  *status = v;
  return B2_OK;
}

int b2_jk_status(int reset, int *status) {
  if (!status) return B2_ERR_ARG;
  const int v = b2_jk_status_read(reset);
  if (v < 0) return B2_ERR_CUDA;
  *status = v;
  return B2_OK;
}

int b2_plan_set_subset(void *plan, const int *mols, int n) {
  if (!plan || n < 0 || (n > 0 && !mols)) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  b2_subset_free(P);
  if (n == 0) return B2_OK;
  if (P->g.xblk32_h.empty()) return B2_ERR_ARG;
  std::vector<int> map(mols, mols + n);
  std::vector<long long> jo(n + 1, 0), x3(n + 1, 0), x6(n + 1, 0), xt(n + 1, 0), so(n + 1, 0);
  for (int k = 0; k < n; ++k) {
    const int m = map[k];
    if (m < 0 || m >= P->h.nmol) return B2_ERR_ARG;
    jo[k + 1] = jo[k] + (P->jk_off_h[m + 1] - P->jk_off_h[m]);
    x3[k + 1] = x3[k] + (P->g.xblk32_h[m + 1] - P->g.xblk32_h[m]);
    x6[k + 1] = x6[k] + (P->g.xblk64_h[m + 1] - P->g.xblk64_h[m]);
    xt[k + 1] = xt[k] + (P->g.xblk_tc_h[m + 1] - P->g.xblk_tc_h[m]);
    so[k + 1] = so[k] + (P->sv_off_h[m + 1] - P->sv_off_h[m]);
  }
  int rc;
  if ((rc = b2_upload(&P->sub.mol_map, map)) || (rc = b2_upload(&P->sub.jk_off, jo)) ||
      (rc = b2_upload(&P->sub.x32, x3)) || (rc = b2_upload(&P->sub.x64, x6)) ||
      (rc = b2_upload(&P->sub.xtc, xt)) || (rc = b2_upload(&P->sub.sv_off, so))) {
    b2_subset_free(P);
    return rc;
  }
  P->sub.n = n;
  P->sub.jk_n = jo[n];
  P->sub.n_x32 = x3[n];
  P->sub.n_x64 = x6[n];
  P->sub.n_xtc = xt[n];
  P->sub.sv_n = so[n];
  std::vector<int> bmap;
  b2_buckets(P, map, bmap, P->sub.bkt_off_h);
  if ((rc = b2_upload(&P->sub.bkt_map, bmap)) || (rc = b2_xq_build(*P, map, &P->sub.xq_items, P->sub.xq_off_h))) {
    b2_subset_free(P);
    return rc;
  }
  return B2_OK;
}

int b2_eri_s8(void *plan, int precision, void *eri_out, void *stream) {
  if (!plan || !eri_out) return B2_ERR_ARG;
  int rc = b2_launch_eri_s8(*(B2PlanDev *)plan, precision, eri_out, (cudaStream_t)stream);
  if (rc == B2_ERR_CUDA) b2_note(cudaGetLastError());
  return rc;
}

int b2_jk_exchange(void *plan, int precision, const void *eri, void *exch, void *stream) {
  if (!plan || !eri || !exch) return B2_ERR_ARG;
  return b2_launch_exch_build(*(B2PlanDev *)plan, precision, eri, exch, (cudaStream_t)stream);
}

int b2_jk_pairs(void *plan, int precision, const int *active, const void *eri, const void *exch,
                const double *D, double *J, double *K, void *stream) {
  if (!plan || !eri || !exch || !D || !J || !K) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  return b2_launch_jk_symv(*P, precision, active, eri, exch, D, J, K, P->sv_work, (cudaStream_t)stream);
}

int b2_jk_s8(void *plan, int precision, const int *active, const void *eri, const double *D,
             double *J, double *K, void *stream) {
  if (!plan || !eri || !D || !J || !K) return B2_ERR_ARG;
  return b2_launch_jk_s8(*(B2PlanDev *)plan, precision, active, eri, D, J, K, (cudaStream_t)stream);
}

int b2_grid_set(void *plan, const int64_t *grid_off) {
  if (!plan || !grid_off) return B2_ERR_ARG;
  return b2_grid_setup(*(B2PlanDev *)plan, (const long long *)grid_off);
}

int b2_grid_info(void *plan, int64_t *n_points, int64_t *n_ao) {
  if (!plan) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  if (n_points) *n_points = P->g.n_points;
  if (n_ao) *n_ao = P->g.n_ao;
  return B2_OK;
}

int b2_grid_ao_offsets(void *plan, int64_t *ao_off) {
  if (!plan || !ao_off) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  if (P->g.ao_off_h.empty()) return B2_ERR_ARG;
  for (int m = 0; m < P->h.nmol; ++m) ao_off[m] = P->g.ao_off_h[m];
  return B2_OK;
}

int b2_ao_eval(void *plan, int precision, const double *coords, void *ao, void *stream) {
  if (!plan || !coords || !ao) return B2_ERR_ARG;
  return b2_launch_ao_eval(*(B2PlanDev *)plan, precision, coords, ao, (cudaStream_t)stream);
}

int b2_xc(void *plan, int precision, const int *active, const void *ao, const double *weights,
          const double *D, double *Vxc, double *Exc, void *stream) {
  if (!plan || !ao || !weights || !D || !Vxc || !Exc) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  return b2_launch_xc(*P, precision, active, ao, weights, D, Vxc, Exc, (cudaStream_t)stream);
}

int b2_xc_direct(void *plan, int precision, const int *active, const double *coords,
                 const double *weights, const double *D, double *Vxc, double *Exc, void *stream) {
  if (!plan || !coords || !weights || !D || !Vxc || !Exc) return B2_ERR_ARG;
  return b2_launch_xc_direct(*(B2PlanDev *)plan, precision, active, coords, weights, D, Vxc, Exc,
                             (cudaStream_t)stream);
}

__global__ void k_b3lyp_points(long long n, const double *__restrict__ rho, double *exc,
                               double *vrho, double *vgamma) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  B2XcPoint<double> o = b2_b3lyp_point<double>(rho[g], rho[n + g], rho[2 * n + g], rho[3 * n + g]);
  exc[g] = o.exc; vrho[g] = o.vrho; vgamma[g] = o.vgamma;
}

int b2_b3lyp(int64_t n, const double *rho, double *exc, double *vrho, double *vgamma, void *stream) {
  if (n < 0 || (n > 0 && (!rho || !exc || !vrho || !vgamma))) return B2_ERR_ARG;
  if (n == 0) return B2_OK;
  k_b3lyp_points<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, rho, exc, vrho, vgamma);
  b2_count_launches(1);
  B2_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_chol_inv(void *plan, const double *S, double *Linv, int *status, void *stream) {
  if (!plan || !S || !Linv) return B2_ERR_ARG;
  return b2_launch_chol_inv(*(B2PlanDev *)plan, S, Linv, status, (cudaStream_t)stream);
}

int b2_fock_diis(void *plan, const int *active, const int *iter, double hyb, int use_diis,
                 const double *Hcore, const double *S, const double *D, const double *J,
                 const double *K, const double *Vxc, double *H, double *diffJK, double *ring_err,
                 double *ring_h, double *bmat, double *diis_err, void *stream) {
  if (!plan || !Hcore || !S || !D || !J || !K || !Vxc || !H || !diffJK) return B2_ERR_ARG;
  if (use_diis && (!iter || !ring_err || !ring_h || !bmat || !diis_err)) return B2_ERR_ARG;
  return b2_launch_fock_diis(*(B2PlanDev *)plan, active, iter, hyb, use_diis, Hcore, S, D, J, K,
                             Vxc, H, diffJK, ring_err, ring_h, bmat, diis_err, (cudaStream_t)stream);
}

int b2_eigh_density(void *plan, const int *active, const int *iter, const double *H,
                    const double *Linv, double *D, double *mo_energy, double *C, double *ws,
                    int *sweeps, void *stream) {
  if (!plan || !H || !Linv || !D || !mo_energy) return B2_ERR_ARG;
  return b2_launch_eigh_density(*(B2PlanDev *)plan, active, iter, H, Linv, D, mo_energy, C, ws,
                                sweeps, (cudaStream_t)stream);
}

int b2_energy(void *plan, const int *active, const double *D, const double *Hcore,
              const double *diffJK, const double *Exc, const double *Enuc, double *out,
              void *stream) {
  if (!plan || !D || !Hcore || !diffJK || !Exc || !Enuc || !out) return B2_ERR_ARG;
  return b2_launch_energy(*(B2PlanDev *)plan, active, D, Hcore, diffJK, Exc, Enuc, out,
                          (cudaStream_t)stream);
}

int b2_fp32_peak(double *tflops) {
  if (!tflops) return B2_ERR_ARG;
  return b2_measure_fp32_peak(tflops);
}

int b2_eri_work(void *plan, double *out) {
  if (!plan || !out) return B2_ERR_ARG;
  return b2_launch_eri_count(*(B2PlanDev *)plan, out);
}

int b2_copy_blocks(int n, const void *src, void *dst, const int64_t *src_off, const int64_t *dst_off,
                   const int64_t *len, void *stream) {
  if (n < 0 || (n > 0 && (!src || !dst || !src_off || !dst_off || !len))) return B2_ERR_ARG;
  return b2_launch_copy_blocks(n, src, dst, (const long long *)src_off, (const long long *)dst_off,
                               (const long long *)len, (cudaStream_t)stream);
}

int b2_scf_iterate(void *plan, const b2_scf_state *S, void *stream) {
  if (!plan || !S) return B2_ERR_ARG;
  if (!S->Hcore || !S->S || !S->Linv || !S->weights || !S->enuc || !S->eri || !S->D || !S->J || !S->K ||
      !S->Vxc || !S->H || !S->diffJK || !S->ring_err || !S->ring_h || !S->bmat || !S->diis_err || !S->exc ||
      !S->energy || !S->mo_energy || !S->iter || !S->active || (!S->ao && !S->coords))
    return B2_ERR_ARG;
  if (S->precision != 64 && S->precision != 32) return B2_ERR_ARG;
  B2PlanDev &P = *(B2PlanDev *)plan;
  cudaStream_t st = (cudaStream_t)stream;
  const int *a = S->active;
  int rc = b2_launch_fock_diis(P, a, S->iter, S->hyb, S->use_diis, S->Hcore, S->S, S->D, S->J, S->K,
                               S->Vxc, S->H, S->diffJK, S->ring_err, S->ring_h, S->bmat, S->diis_err, st);
  if (!rc) rc = b2_launch_eigh_density(P, a, S->iter, S->H, S->Linv, S->D, S->mo_energy, S->C, S->eig_ws,
                                       S->sweeps, st);
  // XC (issue-bound, on the bucket streams forked from st) and J/K (HBM-bound) both read only the
  // new density: J/K runs beside XC on the plan's J/K stream, forked after the eigensolver and
  // joined before the energies
  cudaStream_t js = P.jk_stream ? P.jk_stream : st;
  if (!rc && js != st) {
    rc = b2_note(cudaEventRecord(P.jk_ev[0], st));
    if (!rc) rc = b2_note(cudaStreamWaitEvent(js, P.jk_ev[0], 0));
  }
  if (!rc) rc = S->ao ? b2_launch_xc(P, S->precision, a, S->ao, S->weights, S->D, S->Vxc, S->exc, st)
                      : b2_launch_xc_direct(P, S->precision, a, S->coords, S->weights, S->D, S->Vxc, S->exc, st);
  if (!rc) rc = S->exch ? b2_launch_jk_symv(P, S->precision, a, S->eri, S->exch, S->D, S->J, S->K, P.sv_work, js)
                        : b2_launch_jk_s8(P, S->precision, a, S->eri, S->D, S->J, S->K, js);
  if (!rc && js != st) {
    rc = b2_note(cudaEventRecord(P.jk_ev[1], js));
    if (!rc) rc = b2_note(cudaStreamWaitEvent(st, P.jk_ev[1], 0));
  }
  if (!rc) rc = b2_launch_energy_jk(P, a, S->D, S->Hcore, S->J, S->K, S->hyb, S->exc, S->enuc, S->diffJK,
                                    S->energy, S->iter, st);
  return rc;
}

int b2_int2e_sph_s8(const int *atm, int natm, const int *bas, int nbas, const double *env,
                    int n_env, int precision, void *eri_out, void *stream) {
  if (!atm || !bas || !env || !eri_out || natm <= 0 || nbas <= 0 || n_env <= 0) return B2_ERR_ARG;
  int64_t eo = 0;
  void *plan = nullptr;
  int rc = b2_plan_create(1, &natm, &nbas, atm, bas, env, &eo, &plan);
  if (rc) return rc;
  rc = b2_eri_s8(plan, precision, eri_out, stream);
  if (!rc) rc = b2_note(cudaStreamSynchronize((cudaStream_t)stream));
  b2_plan_destroy(plan);
  return rc;
}

int b2_int1e(void *plan, double *S, double *T, double *V, void *stream) {
  if (!plan || !S || !T || !V) return B2_ERR_ARG;
  return b2_launch_int1e(*(B2PlanDev *)plan, S, T, V, (cudaStream_t)stream);
}

int b2_grid_build(void *plan, int nz, const double *tmpl, const int64_t *tmpl_off, double *coords,
                  double *weights, void *stream) {
  if (!plan || !tmpl || !tmpl_off || !coords || !weights) return B2_ERR_ARG;
  return b2_launch_grid_build(*(B2PlanDev *)plan, nz, tmpl, (const long long *)tmpl_off, coords,
                              weights, (cudaStream_t)stream);
}

int b2_guess(void *plan, double *D, void *stream) {
  if (!plan || !D) return B2_ERR_ARG;
  return b2_launch_guess(*(B2PlanDev *)plan, D, (cudaStream_t)stream);
}

int b2_enuc(void *plan, double *enuc, void *stream) {
  if (!plan || !enuc) return B2_ERR_ARG;
  return b2_launch_enuc(*(B2PlanDev *)plan, enuc, (cudaStream_t)stream);
}

int b2_eri_threshold(void *plan, int precision, void *eri, double threshold, void *stream) {
  if (!plan) return B2_ERR_ARG;
  return b2_launch_eri_threshold(*(B2PlanDev *)plan, precision, eri, threshold, (cudaStream_t)stream);
}

int b2_grad(void *plan, int parts, double hyb, const double *C, const double *mo_energy, const double *coords,
            const double *weights, double *D, double *W, double *grad, void *stream) {
  if (!plan) return B2_ERR_ARG;
  B2PlanDev *P = (B2PlanDev *)plan;
  if (P->h.max_natm > B2_MAXNAO) return B2_ERR_SIZE;
  return b2_launch_grad(*P, parts, hyb, C, mo_energy, coords, weights, D, W, grad, (cudaStream_t)stream);
}

}  // extern "C"
