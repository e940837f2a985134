// Device copy of a batch plan (owned by the C-ABI plan handle).
#pragma once
#include "plan_host.hpp"
#include "boys.cuh"
#include "eri_sq.cuh"

// number of kernels this library has launched (monotonic; read with b2_launch_count)
void b2_count_launches(long long n);

#define B2_NBKT 5              // orbital buckets nao <= 16, 32, 48, 64, more

struct B2GridDev {             // grid layout registered with b2_grid_set
  long long n_points = 0, n_gblk = 0, n_xblk32 = 0, n_xblk64 = 0, n_xblk_tc = 0, n_ao = 0;
  long long *grid_off = nullptr, *gblk_off = nullptr, *ao_off = nullptr;
  long long *xblk32 = nullptr, *xblk64 = nullptr;   // fused-XC CTA prefix per precision
  long long *xblk_tc = nullptr;                     // tensor-core XC CTA prefix (128-point tiles)
  int tpc32 = 1, tpc64 = 1, tpc_tc = 1;             // tiles per CTA
  double *tmpl = nullptr;      // atomic grid templates (x, y, z, w)
  long long *tmpl_off = nullptr, *atom_pt_off = nullptr;
  std::vector<long long> grid_off_h, ao_off_h, xblk32_h, xblk64_h, xblk_tc_h;
  void *xq_items = nullptr;                         // per-bucket XC work items (molecule, tile)
  std::vector<long long> xq_off_h;                  // B2_NBKT + 1 bucket starts in xq_items
  int *xq_queue = nullptr;                          // B2_NBKT work-queue counters
  int xq_tpc[B2_NBKT] = {0, 0, 0, 0, 0};            // tiles per item per bucket (0: tpc_tc)
};

struct B2SubsetDev {           // compacted work tables for a subset of the batch's molecules
  int n = 0;                   // 0: no subset (full tables)
  int *mol_map = nullptr;      // compacted index -> molecule
  int *bkt_map = nullptr;      // the subset's molecules by orbital bucket
  std::vector<int> bkt_off_h;  // B2_NBKT + 1
  long long *jk_off = nullptr, *x32 = nullptr, *x64 = nullptr, *xtc = nullptr, *sv_off = nullptr;
  long long jk_n = 0, n_x32 = 0, n_x64 = 0, n_xtc = 0, sv_n = 0;
  void *xq_items = nullptr;    // per-bucket XC work items of the subset
  std::vector<long long> xq_off_h;
};

struct B2PlanDev {
  B2PlanHost h;
  B2MolDev *mols = nullptr;
  long long *row_off = nullptr;
  B2Shell *shells = nullptr;
  B2PairInfo *pinfo = nullptr;
  B2PairPrim<double> *pp64 = nullptr;
  B2PairPrim<float> *pp32 = nullptr;
  unsigned char *pp32_n = nullptr;        // per shell pair: surviving float32 primitive pairs
  int *ao2sh = nullptr;
  int *cls_list = nullptr;
  int *cls_cnt = nullptr;
  double *atom_xyz = nullptr;
  int *atom_z = nullptr;
  double *boys = nullptr;
  float *boys32 = nullptr;                // float copy for the float32 kernels
  long long *jk_chunk_off = nullptr;      // nmol + 1 (J/K work split)
  long long jk_chunk = 0;
  long long jk_nchunks = 0;
  int device = 0;
  long long h2d_bytes = 0;                // bytes copied host -> device by plan creation
  B2GridDev g;
  B2EriTask *eri_tasks32 = nullptr, *eri_tasks64 = nullptr;
  std::vector<long long> eri_goff32, eri_goff64;   // task group (class combination) starts
  std::vector<long long> jk_off_h;                 // host copy of jk_chunk_off
  B2SubsetDev sub;
  int xc_impl = 0;             // float32 XC: 0 = tensor-core kernel, 1 = SIMT kernel
  long long *sv_off = nullptr;            // nmol + 1: warp tasks of the J/K products per molecule
  std::vector<long long> sv_off_h;
  long long sv_ntask = 0;
  double *sv_work = nullptr;              // 4 x n_rows: x_J, x_K, y_J, y_K
  int *bkt_map = nullptr;                 // molecules ordered by orbital bucket
  std::vector<int> bkt_map_h;
  std::vector<int> bkt_off_h;             // B2_NBKT + 1 bucket starts in bkt_map
  cudaStream_t bkt_stream[B2_NBKT] = {};  // per-bucket streams (forked from / joined to the caller's)
  cudaEvent_t bkt_ev[B2_NBKT + 1] = {};
  cudaStream_t jk_stream = nullptr;       // J/K beside XC in an SCF iteration (forked / joined)
  cudaEvent_t jk_ev[2] = {};
};

int b2_launch_eri_s8(B2PlanDev &P, int precision, void *out, cudaStream_t st);
// the ERI work list of `precision` (32: canonical shell quartets grouped by class combination,
// up to 32 kets per task; 64: p-shell bras split by component), built once per plan
int b2_eri_tasks_ready(B2PlanDev &P, int precision, cudaStream_t st);
int b2_launch_grad(B2PlanDev &P, int parts, double hyb, const double *C, const double *mo_energy,
                   const double *coords, const double *weights, double *D, double *W, double *grad,
                   cudaStream_t st);
int b2_build_pairs(B2PlanDev &P, cudaStream_t st);
int b2_launch_exch_build(const B2PlanDev &P, int precision, const void *eri, void *exch, cudaStream_t st);
int b2_launch_jk_symv(const B2PlanDev &P, int precision, const int *active, const void *eri,
                      const void *exch, const double *D, double *J, double *K, double *work,
                      cudaStream_t st);
long long b2_sv_tasks_host(long long n2);
int b2_jk_status_read(int reset);     // error flag of the J/K product kernel (-1: CUDA error)
int b2_launch_jk_s8(const B2PlanDev &P, int precision, const int *active, const void *eri,
                    const double *D, double *J, double *K, cudaStream_t st);
int b2_zero_active(const B2PlanDev &P, const int *active, double *A, double *B, cudaStream_t st);
// per-bucket work items of the tensor-core XC kernel for `mols` (device array in *items,
// bucket starts in off), P.g.tpc_tc tiles per item
int b2_xq_build(const B2PlanDev &P, const std::vector<int> &mols, void **items, std::vector<long long> &off);
// measurement and slot-refill helpers (eri.cu, blocks.cu)
int b2_launch_eri_count(B2PlanDev &P, double *host_out);
int b2_measure_fp32_peak(double *tflops);
int b2_launch_copy_blocks(int n, const void *src, void *dst, const long long *src_off,
                          const long long *dst_off, const long long *len, cudaStream_t st);
