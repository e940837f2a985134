/* b200dft C ABI: B200 (sm_100a) kernels for the restricted Kohn-Sham SCF hot path of
 * pyscf-ipu.  Plain C types only.  Device buffers are caller-owned device pointers;
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  Every
 * function returns 0 on success or a negative B2_ERR_* code; nothing throws across the ABI.
 *
 * Molecules enter as the libcint atm/bas/env arrays that the reference packs for its own
 * native ERI code (pyscf_ipu/electron_repulsion/direct.py:710-739 prepare_int_floats /
 * prepare_integrals_2_inputs; consumed by int2e_sph, int2e_sph.cpp:6750).  A batch is the
 * concatenation of each molecule's atm rows (6 ints), bas rows (8 ints) and env segment;
 * pointers inside atm/bas are relative to the molecule's env segment (env_off[m]).
 *
 * Per-molecule device layouts (offsets from b2_plan_offsets):
 *   s8 ERIs:   eri_off[m] + ij(ij+1)/2 + kl, ij = i(i+1)/2 + j, i>=j, k>=l, ij>=kl
 *   matrices:  mat_off[m] + a*nao + b (row-major nao x nao, float64)
 *   AO values: ao_off[m] + (c*G + g)*nao + n, c = value, d/dx, d/dy, d/dz
 *   grid:      grid_off[m] + g (coords: 3 doubles per point)
 */
#ifndef B200DFT_H
#define B200DFT_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define B2_OK 0
#define B2_ERR_ARG (-1)
#define B2_ERR_CUDA (-2)
#define B2_ERR_UNSUPPORTED (-3)
#define B2_ERR_SIZE (-4)
#define B2_ERR_NOT_PD (-5)
#define B2_ERR_TIMEOUT (-6)

typedef void *b2_plan_t;

/* Library/ABI version (major*10000 + minor*100 + patch). */
int b2_version(void);

/* Number of kernels the library has launched in this process (monotonic counter; kernels
 * replayed from a captured CUDA graph are not counted again). */
int b2_launch_count(int64_t *out);

/* Last CUDA error string seen by the library (for diagnostics). */
const char *b2_last_error(void);

/* Build a batch plan from host libcint arrays and upload its tables to the current device.
 * Replaces the host preparation of the reference's ERI path: prepare_int_floats and
 * prepare_integrals_2_inputs (electron_repulsion/direct.py:710-944). */
int b2_plan_create(int nmol, const int *natm, const int *nbas, const int *atm, const int *bas,
                   const double *env, const int64_t *env_off, b2_plan_t *plan);
int b2_plan_destroy(b2_plan_t plan);

/* info[0..7] = n_eri_total, n_mat_total, nmol, max_nao, n_rows_total, n_shell_pairs,
 *              jk_chunk, jk_nchunks */
int b2_plan_info(b2_plan_t plan, int64_t *info);

/* Plans and grid tables take device memory from a per-device pool that keeps freed blocks for
 * the next plan (no device synchronisation between batches).  This returns the pool's unused
 * blocks to the driver. */
int b2_release_cached_memory(void);

/* Bytes plan creation copied host -> device (its tables, staged in pinned host memory). */
int b2_plan_h2d_bytes(b2_plan_t plan, int64_t *bytes);

/* Host copies of per-molecule offsets/sizes (arrays of nmol). */
int b2_plan_offsets(b2_plan_t plan, int64_t *eri_off, int64_t *mat_off, int *nao, int *nocc);

/* Re-split the J/K work: `elems` s8 entries per CTA (0 = default policy). */
int b2_plan_set_jk_chunk(b2_plan_t plan, int64_t elems);
/* Float32 exchange-correlation implementation used by b2_xc_direct(precision 32):
 * 0 = per-bucket persistent tcgen05 kernel with TMEM accumulators (default), 1 = CUDA-core
 * kernel, 2 = one-launch tcgen05 kernel.
 * No reference counterpart (replaces the XC einsums of nanoDFT.py:105-123). */
int b2_plan_set_xc_impl(b2_plan_t plan, int impl);
/* Grid tiles (128 points) per CTA of the tensor-core XC kernel; 0 restores the automatic
 * choice.  Clears any molecule subset set with b2_plan_set_subset.  No reference counterpart. */
int b2_plan_set_xc_tiles(b2_plan_t plan, int tiles_per_cta);
/* Grid tiles per work item of the per-bucket tensor-core XC kernel, one value per orbital bucket
 * (host int[5]: nao <= 16, 32, 48, 64, more; 0 = the plan-wide value).  Set by the autotuner
 * (b200dft.autotune).  Clears any molecule subset.  No reference counterpart. */
int b2_plan_set_xc_bucket_tiles(b2_plan_t plan, const int *tiles);
/* Error code of the tensor-core XC kernel's bounded waits (0 = none); reset != 0 clears it. */
int b2_xc_tc_status(int reset, int *status);

/* Error flag of the J/K product kernel's copy waits (0 = none; 1 = a wait on a row-group
 * copy gave up and that warp's contribution is missing); reset != 0 clears it after reading. */
int b2_jk_status(int reset, int *status);

/* Restrict the J/K and XC launches to a subset of the batch's molecules (host int[n] molecule
 * indices; n = 0 restores the full batch).  Used when few molecules are still iterating, so the
 * launches cover only their work. */
int b2_plan_set_subset(b2_plan_t plan, const int *mols, int n);

/* All unique ERIs of every molecule into the s8 layout, precision 64 (float64 out) or 32
 * (float32 out).  Replaces int2e_sph (int2e_sph.cpp:6750) dispatched per shell quartet by
 * compute_integrals_2 / integrals_v1 (direct.py:506-707), and mol.intor('int2e_sph',
 * aosym='s8') (nanoDFT.py:285). */
int b2_eri_s8(b2_plan_t plan, int precision, void *eri_out, void *stream);

/* J and K (float64, nao x nao per molecule) from the s8 list and D (float64).  Arithmetic in
 * `precision` (64 or 32, must match the ERI buffer).  Replaces sparse_symmetric_einsum
 * (nanoDFT/sparse_symmetric_ERI.py:86) and ipu_direct_mult (electron_repulsion/direct.py:489);
 * diff_JK = J - K*hyb/2 as in get_JK (nanoDFT.py:125-139).  active: device int[nmol] or NULL;
 * molecules with active[m] == 0 are skipped and their J/K left untouched. */
int b2_jk_s8(b2_plan_t plan, int precision, const int *active, const void *eri, const double *D,
             double *J, double *K, void *stream);

/* Exchange list of a batch's s8 ERI list: H[(il),(jk)] = (ij|kl) + (ik|jl) for pairs i >= l,
 * j >= k, packed like the s8 list (same offsets and size; precision 64: double, 32: float).
 * Build once per ERI list; b2_jk_pairs reads both lists.  No counterpart in the reference
 * (an equivalent regrouping of the sums of sparse_symmetric_ERI.py:86-137). */
int b2_jk_exchange(b2_plan_t plan, int precision, const void *eri, void *exch, void *stream);
/* J and K as b2_jk_s8, computed as two symmetric matrix-vector products over the s8 list and
 * the exchange list (float64 arithmetic, no shared-memory atomics).  Both lists must start
 * 16-byte aligned (B2_ERR_ARG otherwise) and hold the plan's padded layout (n_eri_total
 * entries).  Uses a plan-owned workspace: one call at a time per plan. */
int b2_jk_pairs(b2_plan_t plan, int precision, const int *active, const void *eri,
                const void *exch, const double *D, double *J, double *K, void *stream);

/* Register the grid layout: grid_off (host, nmol+1 prefix of per-molecule point counts).
 * Allocates the plan's grid tables and XC scratch on the device. */
int b2_grid_set(b2_plan_t plan, const int64_t *grid_off);
/* Size (elements) of the AO buffer for the registered grid: sum_m 4*G_m*nao_m. */
int b2_grid_info(b2_plan_t plan, int64_t *n_points, int64_t *n_ao);
int b2_grid_ao_offsets(b2_plan_t plan, int64_t *ao_off);

/* AO values and gradients on the grid (replaces mol.eval_gto('GTOval_sph_deriv1', coords, 4),
 * dft.py:220).  coords: device float64 (n_points x 3); ao: device, precision 64 or 32. */
int b2_ao_eval(b2_plan_t plan, int precision, const double *coords, void *ao, void *stream);

/* E_xc (nmol float64) and symmetric V_xc (float64 matrices) for densities D; replaces
 * exchange_correlation (nanoDFT.py:105-123) / xc (dft.py:899-1036) minus the J/K part. */
int b2_xc(b2_plan_t plan, int precision, const int *active, const void *ao,
          const double *weights, const double *D, double *Vxc, double *Exc, void *stream);

/* As b2_xc, with AO values and gradients generated on the fly per tile of grid points from
 * the basis (no stored AO tensor); coords: device float64 (n_points x 3). */
int b2_xc_direct(b2_plan_t plan, int precision, const int *active, const double *coords,
                 const double *weights, const double *D, double *Vxc, double *Exc, void *stream);

/* B3LYP at n points: rho (4 x n, device float64, rho[1:4] = half density gradient as the
 * reference forms it) -> e_xc, vrho, vgamma (device float64).  Replaces b3lyp(rho, eps)
 * (exchange_correlation/b3lyp.py:13). */
int b2_b3lyp(int64_t n, const double *rho, double *exc, double *vrho, double *vgamma,
             void *stream);

/* L = inv(cholesky(S)) per molecule (dft.py:234, nanoDFT.py:239); status[m] = 0 or
 * B2_ERR_NOT_PD (device int array, may be NULL). */
int b2_chol_inv(b2_plan_t plan, const double *S, double *Linv, int *status, void *stream);

/* One Fock build + DIIS step per molecule (nanoDFT.py:63-66, DIIS 338-364).  active (device
 * int[nmol] or NULL = all), iter (device int[nmol]: the molecule's iteration index).
 * ring_err / ring_h: device float64, 9 * n_mat each; bmat: device float64 100 * nmol;
 * diis_err: device float64 [nmol] (max |SDH - HDS|). */
int b2_fock_diis(b2_plan_t plan, const int *active, const int *iter, double hyb, int use_diis,
                 const double *Hcore, const double *S, const double *D, const double *J,
                 const double *K, const double *Vxc, double *H, double *diffJK, double *ring_err,
                 double *ring_h, double *bmat, double *diis_err, void *stream);

/* C = L^T eigvec(L H L^T), D = 2 C_occ C_occ^T (nanoDFT.py:68-72).  mo_energy: device float64
 * nmol x 72 (ascending, first nao valid); C may be NULL; sweeps (device int[nmol]) may be NULL.
 * ws (device float64 n_mat, may be NULL): eigenvector basis kept between calls; with iter[m] > 0
 * the solve starts from it (warm start), with iter NULL or iter[m] == 0 it starts cold. */
int b2_eigh_density(b2_plan_t plan, const int *active, const int *iter, const double *H,
                    const double *Linv, double *D, double *mo_energy, double *C, double *ws,
                    int *sweeps, void *stream);

/* energies (device float64 nmol x 5): [E, E_core, E_J_K/2, E_xc, E_nuc] (nanoDFT.py:20-38) */
int b2_energy(b2_plan_t plan, const int *active, const double *D, const double *Hcore,
              const double *diffJK, const double *Exc, const double *Enuc, double *out,
              void *stream);

/* One-electron matrices S, T, V (float64 matrices) for every molecule; replaces
 * mol.intor_symmetric('int1e_ovlp' / 'int1e_kin' / 'int1e_nuc') (dft.py:225-227). */
int b2_int1e(b2_plan_t plan, double *S, double *T, double *V, void *stream);

/* Becke-partitioned grid for every molecule (replaces Grids(mol).build(), dft.py:214-216 and
 * pyscf_utils/build_grid.py:109-135).  tmpl: host float64 (x, y, z, w) per template point of
 * each element's atom-centred grid, tmpl_off: host prefix (nz+1) indexed by nuclear charge.
 * The layout registered by b2_grid_set must equal the sum of the atoms' template sizes.
 * coords (n_points x 3) and weights (n_points): device float64. */
int b2_grid_build(b2_plan_t plan, int nz, const double *tmpl, const int64_t *tmpl_off,
                  double *coords, double *weights, void *stream);

/* MINAO-style initial density (atomic occupations on the diagonal; minao, dft.py:223). */
int b2_guess(b2_plan_t plan, double *D, void *stream);

/* Nuclear repulsion per molecule (mol.energy_nuc(), dft.py:202); device float64 [nmol]. */
int b2_enuc(b2_plan_t plan, double *enuc, void *stream);

/* ERI threshold (nanoDFT.py:280-288, option eri_threshold): every entry of the s8 list with
 * |v| <= threshold becomes 0.  Apply before b2_jk_exchange, which reads the thresholded list. */
int b2_eri_threshold(b2_plan_t plan, int precision, void *eri, double threshold, void *stream);

/* Nuclear gradient of converged SCFs, float64 (replaces grad(mol, coords, weight, mo_coeff,
 * mo_energy) = grad_elec + grad_nuc, nanoDFT.py:403-477, with the grid held fixed as there).
 * With C (device float64 matrices at the plan's matrix offsets, column k = orbital k) and
 * mo_energy (device float64 nmol x 72), D and W (caller-owned device matrices) receive
 * dm0 = 2 C_occ C_occ^T and dme0 = 2 C_occ eps_occ C_occ^T; with C NULL they are inputs.
 * grad (device float64, 3 per atom, each molecule's atoms from its atom offset = the sum of
 * natm of the molecules before it) is overwritten with the sum of the parts selected by
 * `parts`: bit 0 one-electron (kinetic, nuclear attraction, -<dme0, dS>), bit 1 two-electron
 * (Coulomb and hyb-scaled exchange), bit 2 exchange-correlation (B3LYP on coords / weights, the
 * layout registered with b2_grid_set), bit 3 nuclear repulsion; 15 = the full gradient.
 * hyb: exact-exchange fraction (0.2 for B3LYP).  Not for graph capture: the exchange-correlation
 * part copies a small host table per call, and the first call on a plan that has not built its
 * float32 ERI work list builds it, synchronising `stream`. */
int b2_grad(b2_plan_t plan, int parts, double hyb, const double *C, const double *mo_energy,
            const double *coords, const double *weights, double *D, double *W, double *grad,
            void *stream);

/* Device buffers of a batch's SCF state for b2_scf_iterate (all nmol molecules of the plan,
 * layouts as for the entries above; matrices float64 at the plan's matrix offsets).
 * Inputs: Hcore, S, Linv; weights and either coords (AO values generated per grid tile) or ao
 * (stored AO values, precision `precision`); enuc [nmol]; eri (s8 list, `precision`) and exch
 * (its exchange list, or NULL to contract the s8 list directly).  State carried between
 * iterations: D, J, K, Vxc, H, diffJK, ring_err / ring_h (9 n_mat each), bmat (100 nmol),
 * diis_err, exc, energy (5 nmol), mo_energy (72 nmol), C and eig_ws (may be NULL), iter, active
 * (int nmol; molecules with active == 0 are skipped), sweeps (may be NULL). */
typedef struct {
  const double *Hcore, *S, *Linv, *coords, *weights, *enuc;
  const void *ao, *eri, *exch;
  double *D, *J, *K, *Vxc, *H, *diffJK, *ring_err, *ring_h, *bmat, *diis_err, *exc, *energy, *mo_energy, *C,
      *eig_ws;
  int *iter, *active, *sweeps;
  double hyb;
  int use_diis, precision;
} b2_scf_state;

/* One SCF iteration of every active molecule (nanoDFT_iteration, nanoDFT.py:40-102): Fock build
 * + DIIS, orthogonalised eigensolve and new density, V_xc / E_xc, J / K, diff_JK = J - hyb/2 K,
 * the five energy terms, iter += 1.  Launches kernels only (on `stream` and the plan's bucket
 * streams, joined back to `stream`), so a call can be captured into a CUDA graph and replayed;
 * one capture serves every later iteration. */
int b2_scf_iterate(b2_plan_t plan, const b2_scf_state *state, void *stream);

/* Work of the float32 ERI kernels for this plan (measurement; synchronises the device): out[0] =
 * primitive quartets evaluated (surviving bra x ket primitive pairs of every shell quartet),
 * out[1] = their arithmetic by the per-class counts generated from the kernels' own code
 * (csrc/eri_flops.h), out[2] = their special-function operations.  No reference counterpart. */
int b2_eri_work(b2_plan_t plan, double *out);

/* Measured FP32 FMA rate of the current GPU in TFLOP/s (every SM full of threads running
 * independent FMA chains; CUDA events around one launch; synchronises the device).  The
 * denominator of the ERI kernels' roofline fraction.  No reference counterpart. */
int b2_fp32_peak(double *tflops);

/* n block copies dst[dst_off[k] .. + len[k]) = src[src_off[k] .. + len[k]) (bytes; the offset and
 * length arrays are device int64[n]).  Carries the state of molecules still iterating (their
 * s8 and exchange lists) into the layout of the plan that refills the batch's converged slots.
 * No reference counterpart. */
int b2_copy_blocks(int n, const void *src, void *dst, const int64_t *src_off, const int64_t *dst_off,
                   const int64_t *len, void *stream);

/* Single-molecule convenience mirroring the reference's native entry int2e_sph
 * (int2e_sph.cpp:6750): host libcint arrays in, all s8 ERIs of the molecule out (device). */
int b2_int2e_sph_s8(const int *atm, int natm, const int *bas, int nbas, const double *env,
                    int n_env, int precision, void *eri_out, void *stream);

/* Allocation-free single-molecule ERI entry (no counterpart in the reference).  For callers
 * that must not call cudaMalloc: processes whose device memory is handed out by another
 * allocator or a fixed-budget pool, and loops with a latency budget (cudaMalloc/cudaFree can
 * block and synchronise the device).  Same inputs and s8 output as b2_int2e_sph_s8, but the
 * tables live in a 2.5 MiB static device array that every GPU loading the library keeps until
 * exit.  Limits: nbas <= 48 shells, nao <= 70 (B2_ERR_SIZE beyond).  Unlike b2_int2e_sph_s8 it
 * does not synchronise: the output is ready, and kernel errors show, only after the caller
 * synchronises `stream`.  All calls share the static array and a static host staging buffer:
 * calls from several host threads must be serialised by the caller, and calls whose work
 * overlaps on the GPU (different streams) race; calls on one stream are ordered.  The first
 * call on a device looks up the array's address with that device current; make it before any
 * stream capture. */
int b2_int2e_sph_s8_noalloc(const int *atm, int natm, const int *bas, int nbas, const double *env,
                            int n_env, int precision, void *eri_out, void *stream);

/* ---- Learned initial guess: kernels of the message-passing network that predicts D0 ----
 * No counterpart in the reference's code (its nanoDFT README describes the learned guess as
 * future work; the reference runs minao, pyscf_utils/minao.py:5-123).  Float32 device
 * buffers; every call takes the stream to launch on and returns B2_OK or an error code.
 * Forward and backward of one training step and the prediction are compositions of these. */

/* C[M,N] = beta*C + A B (+ bias[N]); A element (i,k) at A[i*sai + k*sak], B (k,j) at
 * B[k*sbk + j*sbj].  bf16: 0 float32, 1 operands rounded to bfloat16 (CUDA cores),
 * 2 bfloat16 operands on the tcgen05 tensor cores (float32 accumulation in tensor memory). */
int b2_nn_gemm(int M, int N, int K, const float *A, int64_t sai, int64_t sak, const float *B,
               int64_t sbk, int64_t sbj, float *C, int64_t ldc, const float *bias, float beta,
               int bf16, void *stream);
/* *status = 1 if a bounded internal wait of the tcgen05 product gave up since the last reset
 * (that launch left C untouched), else 0; reset != 0 clears it.  Synchronous. */
int b2_nn_gemm_status(int reset, int *status);
/* out[N] (+)= column sums of X[M,N] (row stride ld); accumulate != 0 adds to out. */
int b2_nn_colsum(int M, int N, const float *X, int64_t ld, float *out, int accumulate, void *stream);
/* y = x * sigmoid(x) and its backward dx = dy * silu'(x). */
int b2_nn_silu(int64_t n, const float *x, float *y, void *stream);
int b2_nn_silu_bwd(int64_t n, const float *x, const float *dy, float *dx, void *stream);
/* R Gaussian radial basis functions on [0, rc] of P distances r -> out[P,R]. */
int b2_nn_rbf(int64_t P, int R, float rc, const float *r, float *out, void *stream);
/* Message passing over a CSR graph (ptr by receiving atom, src = sender): out[a,:] (+)=
 * sum_e phi[e,:] * h[src[e],:]. */
int b2_nn_message(int A, int F, const int *ptr, const int *src, const float *phi, const float *h,
                  float *out, int accumulate, void *stream);
/* out[e,:] = dm[dst[e],:] * h[src[e],:] (edge gradient of the message). */
int b2_nn_pairmul(int64_t P, int F, const int *src, const int *dst, const float *dm, const float *h,
                  float *out, void *stream);
/* Pair features x[p] = [h[pa[p]], h[pb[p]], rbf[p]] (width 2F+R) and the transpose of the
 * gather: dh[pa[p]] += dx[p][0:F], dh[pb[p]] += dx[p][F:2F]. */
int b2_nn_gather(int64_t P, int F, int R, const int *pa, const int *pb, const float *h,
                 const float *rbf, float *x, void *stream);
int b2_nn_scatter(int64_t P, int F, int R, const int *pa, const int *pb, const float *dx, float *dh,
                  void *stream);
/* Atom-type embedding h[a,:] = E[type[a],:] and its backward dE. */
int b2_nn_embed(int A, int F, const int *type, const float *E, float *h, void *stream);
int b2_nn_embed_bwd(int A, int F, const int *type, const float *dh, float *dE, void *stream);
/* Symmetric density D (float64, per-molecule blocks at mat_off) from the pair scalars z[P,16]
 * and site scalars y[A,4]; with a target Dt also the mean squared error, the residual R and
 * the gradients dz, dy (Dt == NULL: prediction only). */
int b2_nn_assemble(int64_t P, const int *pa, const int *pb, const float *pu, int A,
                   const void *atoms, const int64_t *mat_off, const int *nao, const float *z,
                   const float *y, double *D, int64_t n_mat, const double *Dt, double *R,
                   float *dz, float *dy, double *loss, void *stream);
/* One Adam step with decoupled weight decay wd (step = 1, 2, ...). */
int b2_nn_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1,
               float b2, float eps, int step, float wd, void *stream);

#ifdef __cplusplus
}
#endif
#endif
