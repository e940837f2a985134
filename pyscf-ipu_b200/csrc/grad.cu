// Nuclear gradients of converged RKS SCFs on the GPU, batched over a plan's molecules: the
// reference's grad(mol, coords, weight, mo_coeff, mo_energy) = grad_elec + grad_nuc
// (nanoDFT.py:403-477), which builds int2e_ip1 / int1e_ip* on the host and contracts them with
// einsums.  Here every term is contracted as it is generated, in float64:
//
//   k_grad_dm   dm0 = 2 C_occ C_occ^T, dme0 = 2 C_occ eps_occ C_occ^T (nanoDFT.py:405-406);
//   k_grad_2e   d/dR of 1/2 <D, J> - hyb/4 <D, K> (the vj / vk terms, nanoDFT.py:416-418): one
//               warp per task of the ERI work list (bra shell pair x up to 32 kets of one
//               class), one canonical shell quartet per lane, class-specialised;
//   k_grad_1e   d/dR of <D, T + V_nuc> - <dme0, S> (h1aos and s1, nanoDFT.py:420-424): one CTA
//               per molecule, one ordered shell pair per thread;
//   k_grad_xc   d/dR of E_xc at fixed density and grid (V_xc, nanoDFT.py:408-415): one CTA per
//               32 grid points of one molecule, AO values, D-products and B3LYP staged in
//               shared memory;
//   k_grad_nuc  nuclear repulsion (grad_nuc, nanoDFT.py:428-438).
//
// The per-term math is grad_math.cuh, the same code the host-check build tests against the
// finite-difference oracle.
#include <algorithm>
#include <vector>
#include "device_plan.cuh"
#include "devmem.cuh"
#include "grad_math.cuh"

#define B2G_TP 32                  // grid points per XC tile (one warp's lanes)
#define B2G_XC_THREADS 256

__global__ void __launch_bounds__(256)
k_grad_dm(const B2MolDev *__restrict__ mols, const double *__restrict__ C, const double *__restrict__ eps,
          double *__restrict__ D, double *__restrict__ W) {
  const int m = blockIdx.x;
  const B2MolDev md = mols[m];
  const int N = md.nao, NN = N * N;
  const double *Cm = C + md.mat_off;
  const double *em = eps + (long long)m * B2_MAXNAO;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    double s = 0, t = 0;
    for (int k = 0; k < md.nocc; ++k) {
      const double p = Cm[a * N + k] * Cm[b * N + k];
      s += p;
      t += p * em[k];
    }
    D[md.mat_off + e] = 2.0 * s;
    W[md.mat_off + e] = 2.0 * t;
  }
}

// Two-electron part over canonical shell quartets (b2g_canonical_quartet): one warp per task of
// the float32 ERI work list, whose group fixes the class.  The list also holds kets KL > IJ of
// the bra's last shell (the s8 writer needs them for the component order); those lanes sit out.
template <int G>
__global__ void __launch_bounds__(128)
k_grad_2e(const B2EriTask *__restrict__ tasks, long long ntask, const B2MolDev *__restrict__ mols,
          const B2PairInfo *__restrict__ pinfo, const int *__restrict__ cls_list,
          const B2Shell *__restrict__ shells, const double *__restrict__ btab, const double *__restrict__ D,
          double hyb, double *__restrict__ grad) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ti = (long long)blockIdx.x * 4 + w;
  if (ti >= ntask) return;                        // whole warp
  const B2EriTask tk = tasks[ti];
  const B2MolDev md = mols[tk.mol];
  const B2PairInfo bp = pinfo[md.sp_off + tk.IJ];
  int KL = -1;
  if (lane < tk.count) KL = cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + lane];
  const bool on = KL >= 0 && KL <= tk.IJ;
  double g4[4][3];
  for (int s = 0; s < 4; ++s) for (int x = 0; x < 3; ++x) g4[s][x] = 0.0;
  int atK = 0, atL = 0;
  if (on) {
    const B2PairInfo kp = pinfo[md.sp_off + KL];
    const B2Shell &c = shells[md.sh_off + kp.I], &d = shells[md.sh_off + kp.J];
    b2g_canonical_quartet<b2g_group_l(G, 0), b2g_group_l(G, 1), b2g_group_l(G, 2), b2g_group_l(G, 3)>(
        shells[md.sh_off + bp.I], shells[md.sh_off + bp.J], c, d, bp.I == bp.J, kp.I == kp.J, KL == tk.IJ,
        D + md.mat_off, md.nao, hyb, btab, g4);
    atK = c.atom;
    atL = d.atom;
  }
  // the bra centres are the warp's: one sum over the lanes, one atomic per component
  double *gm = grad + 3ll * md.atm_off;
  for (int s = 0; s < 2; ++s)
    for (int x = 0; x < 3; ++x) {
      double v = g4[s][x];
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(gm + 3 * shells[md.sh_off + (s ? bp.J : bp.I)].atom + x, v);
    }
  if (on)
    for (int x = 0; x < 3; ++x) {
      atomicAdd(gm + 3 * atK + x, g4[2][x]);
      atomicAdd(gm + 3 * atL + x, g4[3][x]);
    }
}

// One-electron part: each thread one ordered shell pair (I, J) of the CTA's molecule; the terms
// on the nuclei (nuclear attraction moving with the nucleus) and on the pair's centres collect
// in shared memory, then one atomic per component per molecule.
__global__ void __launch_bounds__(128)
k_grad_1e(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
          const double *__restrict__ atom_xyz, const int *__restrict__ atom_z, const double *__restrict__ btab,
          const double *__restrict__ D, const double *__restrict__ W, double *__restrict__ grad) {
  __shared__ double sZ[B2_MAXNAO], sR[3 * B2_MAXNAO], sG[3 * B2_MAXNAO];
  const B2MolDev md = mols[blockIdx.x];
  const int natm = md.natm, nbas = md.nbas, N = md.nao;
  for (int e = threadIdx.x; e < natm; e += blockDim.x) sZ[e] = (double)atom_z[md.atm_off + e];
  for (int e = threadIdx.x; e < 3 * natm; e += blockDim.x) {
    sR[e] = atom_xyz[3ll * md.atm_off + e];
    sG[e] = 0.0;
  }
  __syncthreads();
  const double *Dm = D + md.mat_off, *Wm = W + md.mat_off;
  for (int it = threadIdx.x; it < nbas * nbas; it += blockDim.x) {
    const int I = it / nbas, J = it - (it / nbas) * nbas;
    const B2Shell &a = shells[md.sh_off + I], &b = shells[md.sh_off + J];
    double g2[2][3];
    b2g_pair_grad_1e<double>(a, b, Dm, Wm, N, natm, sZ, sR, btab, g2,
                             [&](int c, int x, double v) { atomicAdd(&sG[3 * c + x], v); });
    for (int x = 0; x < 3; ++x) {
      atomicAdd(&sG[3 * a.atom + x], g2[0][x]);
      atomicAdd(&sG[3 * b.atom + x], g2[1][x]);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * natm; e += blockDim.x) atomicAdd(grad + 3ll * md.atm_off + e, sG[e]);
}

// Exchange-correlation part on 32 grid points of one molecule (tile t of molecule m, tile_off:
// per-molecule tile prefix).  With phi the AO values and u = D phi, U_k = D d_k phi:
//   rho = phi.u, grad rho = 2 (d phi).u, and moving atom A moves its orbitals, so
//   dE/dR_A,x = -2 sum_g w sum_{i on A} [vrho d_x phi_i u_i
//                                        + 2 vgamma sum_k g_k (d_x d_k phi_i u_i + d_x phi_i U_k,i)].
// Shared memory: D (N x N), phi and its gradient (4 x N x 32), u and U (4 x N x 32), the
// points' weighted vrho / vgamma and grad rho, and the molecule's atom sums.
__host__ __device__ inline long long b2g_xc_smem_doubles(int N, int natm) {
  return (long long)N * N + 8ll * N * B2G_TP + 5 * B2G_TP + 3ll * natm;
}

__global__ void __launch_bounds__(B2G_XC_THREADS)
k_grad_xc(const B2MolDev *__restrict__ mols, int nmol, const B2Shell *__restrict__ shells,
          const long long *__restrict__ grid_off, const long long *__restrict__ tile_off,
          const double *__restrict__ coords, const double *__restrict__ weights, const double *__restrict__ D,
          double *__restrict__ grad) {
  extern __shared__ double sm[];
  const long long bt = blockIdx.x;
  int lo = 0, hi = nmol - 1;                      // molecule: last m with tile_off[m] <= bt
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_off[mid] <= bt) lo = mid; else hi = mid - 1;
  }
  const int m = lo;
  const B2MolDev md = mols[m];
  const int N = md.nao, nbas = md.nbas, natm = md.natm;
  const long long p0 = grid_off[m] + (bt - tile_off[m]) * B2G_TP;
  const int np = (int)min((long long)B2G_TP, grid_off[m + 1] - p0);
  double *sD = sm;
  double *phi = sD + N * N;                       // [4][N][TP]
  double *u = phi + 4 * N * B2G_TP;               // [4][N][TP]
  double *vr = u + 4 * N * B2G_TP, *vg = vr + B2G_TP, *gr = vg + B2G_TP;   // gr [3][TP]
  double *sG = gr + 3 * B2G_TP;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int e = tid; e < N * N; e += blockDim.x) sD[e] = D[md.mat_off + e];
  for (int e = tid; e < 3 * natm; e += blockDim.x) sG[e] = 0.0;
  // AO values and gradients; item = shell * 32 + point, so a warp shares one shell
  for (int it = tid; it < nbas * B2G_TP; it += blockDim.x) {
    const int s = it / B2G_TP, p = it - s * B2G_TP;
    const B2Shell &S = shells[md.sh_off + s];
    double f[3] = {0, 0, 0}, df[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, hf[3][6];
    if (p < np) b2g_ao2<double>(S, coords + 3 * (p0 + p), f, df, hf);
    for (int c = 0; c < 2 * S.l + 1; ++c) {
      const int i = S.ao0 + c;
      phi[i * B2G_TP + p] = f[c];
      for (int x = 0; x < 3; ++x) phi[((1 + x) * N + i) * B2G_TP + p] = df[c][x];
    }
  }
  __syncthreads();
  for (int it = tid; it < N * B2G_TP; it += blockDim.x) {
    const int i = it / B2G_TP, p = it - i * B2G_TP;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int j = 0; j < N; ++j) {
      const double dij = sD[i * N + j];
      s0 += dij * phi[j * B2G_TP + p];
      s1 += dij * phi[(N + j) * B2G_TP + p];
      s2 += dij * phi[(2 * N + j) * B2G_TP + p];
      s3 += dij * phi[(3 * N + j) * B2G_TP + p];
    }
    u[i * B2G_TP + p] = s0;
    u[(N + i) * B2G_TP + p] = s1;
    u[(2 * N + i) * B2G_TP + p] = s2;
    u[(3 * N + i) * B2G_TP + p] = s3;
  }
  __syncthreads();
  if (tid < B2G_TP) {
    const int p = tid;
    double rho = 0, r1[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i) {
      const double ui = u[i * B2G_TP + p];
      rho += phi[i * B2G_TP + p] * ui;
      for (int x = 0; x < 3; ++x) r1[x] += phi[((1 + x) * N + i) * B2G_TP + p] * ui;
    }
    double a = 0, b = 0;
    if (p < np) {
      const B2XcPoint<double> o = b2_b3lyp_point<double>(rho, r1[0], r1[1], r1[2]);
      const double wt = weights[p0 + p];
      a = wt * o.vrho;
      b = wt * o.vgamma;
    }
    vr[p] = a;
    vg[p] = b;
    for (int x = 0; x < 3; ++x) gr[x * B2G_TP + p] = 2.0 * r1[x];
  }
  __syncthreads();
  const int hidx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  for (int it = tid; it < nbas * B2G_TP; it += blockDim.x) {    // warp-uniform shell
    const int s = it / B2G_TP, p = it - s * B2G_TP;
    const B2Shell &S = shells[md.sh_off + s];
    double acc[3] = {0, 0, 0};
    if (p < np) {
      double f[3], df[3][3], hf[3][6];
      b2g_ao2<double>(S, coords + 3 * (p0 + p), f, df, hf);
      const double a = vr[p], b2 = 2.0 * vg[p];
      const double g0 = gr[p], g1 = gr[B2G_TP + p], g2 = gr[2 * B2G_TP + p];
      for (int c = 0; c < 2 * S.l + 1; ++c) {
        const int i = S.ao0 + c;
        const double u0 = u[i * B2G_TP + p];
        const double uk[3] = {u[(N + i) * B2G_TP + p], u[(2 * N + i) * B2G_TP + p], u[(3 * N + i) * B2G_TP + p]};
        const double gk[3] = {g0, g1, g2};
        for (int x = 0; x < 3; ++x) {
          double q = 0;
          for (int k = 0; k < 3; ++k) q += gk[k] * (hf[c][hidx[x][k]] * u0 + df[c][x] * uk[k]);
          acc[x] += a * df[c][x] * u0 + b2 * q;
        }
      }
    }
    for (int x = 0; x < 3; ++x) {
      double v = acc[x];
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&sG[3 * S.atom + x], -2.0 * v);
    }
  }
  __syncthreads();
  for (int e = tid; e < 3 * natm; e += blockDim.x) atomicAdd(grad + 3ll * md.atm_off + e, sG[e]);
}

// nuclear repulsion: g_a = -sum_{b != a} Z_a Z_b (R_a - R_b) / |R_a - R_b|^3 (coincident atoms
// contribute nothing, as in the reference)
__global__ void __launch_bounds__(128)
k_grad_nuc(const B2MolDev *__restrict__ mols, const double *__restrict__ atom_xyz, const int *__restrict__ atom_z,
           double *__restrict__ grad) {
  const B2MolDev md = mols[blockIdx.x];
  const double *R = atom_xyz + 3ll * md.atm_off;
  const int *Z = atom_z + md.atm_off;
  for (int a = threadIdx.x; a < md.natm; a += blockDim.x) {
    double g[3] = {0, 0, 0};
    for (int b = 0; b < md.natm; ++b) {
      const double d[3] = {R[3 * a] - R[3 * b], R[3 * a + 1] - R[3 * b + 1], R[3 * a + 2] - R[3 * b + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (b == a || r2 == 0.0) continue;
      const double f = (double)Z[a] * Z[b] / (r2 * sqrt(r2));
      for (int x = 0; x < 3; ++x) g[x] -= f * d[x];
    }
    for (int x = 0; x < 3; ++x) atomicAdd(grad + 3ll * (md.atm_off + a) + x, g[x]);
  }
}

template <int G>
static void b2g_launch_2e(const B2PlanDev &P, const double *D, double hyb, double *grad, cudaStream_t st) {
  const long long t0 = P.eri_goff32[G], n = P.eri_goff32[G + 1] - t0;
  if (n > 0) {
    k_grad_2e<G><<<(unsigned)((n + 3) / 4), 128, 0, st>>>(P.eri_tasks32 + t0, n, P.mols, P.pinfo, P.cls_list,
                                                         P.shells, P.boys, D, hyb, grad);
    b2_count_launches(1);
  }
  if constexpr (G < 15) b2g_launch_2e<G + 1>(P, D, hyb, grad, st);
}

int b2_launch_grad(B2PlanDev &P, int parts, double hyb, const double *C, const double *mo_energy,
                   const double *coords, const double *weights, double *D, double *W, double *grad,
                   cudaStream_t st) {
  if (!D || !W || !grad || (parts & ~15)) return B2_ERR_ARG;
  if ((parts & 4) && (!coords || !weights || !P.g.grid_off)) return B2_ERR_ARG;
  const int nmol = P.h.nmol;
  B2_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(double) * 3 * std::max(1, P.h.n_atm), st));
  if (nmol == 0) return B2_OK;
  if (C) {
    if (!mo_energy) return B2_ERR_ARG;
    k_grad_dm<<<nmol, 256, 0, st>>>(P.mols, C, mo_energy, D, W);
    b2_count_launches(1);
  }
  if (parts & 1) {
    k_grad_1e<<<nmol, 128, 0, st>>>(P.mols, P.shells, P.atom_xyz, P.atom_z, P.boys, D, W, grad);
    b2_count_launches(1);
  }
  if (parts & 2) {
    int rc = b2_eri_tasks_ready(P, 32, st);        // canonical quartets grouped by class
    if (rc) return rc;
    b2g_launch_2e<0>(P, D, hyb, grad, st);          // the 16 class combinations
  }
  if (parts & 4) {
    std::vector<long long> toff(nmol + 1, 0);
    for (int m = 0; m < nmol; ++m) {
      const long long G = P.g.grid_off_h[m + 1] - P.g.grid_off_h[m];
      toff[m + 1] = toff[m] + (G + B2G_TP - 1) / B2G_TP;
    }
    if (toff[nmol] > 0) {
      if (toff[nmol] >= (1ll << 31)) return B2_ERR_SIZE;
      const size_t smem = sizeof(double) * (size_t)b2g_xc_smem_doubles(P.h.max_nao, P.h.max_natm);
      B2_CUDA_TRY(cudaFuncSetAttribute(k_grad_xc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      long long *dtoff = nullptr;
      B2_CUDA_TRY(b2_dmalloc_t(&dtoff, sizeof(long long) * (nmol + 1), st));
      // pageable source: the call returns once the data is staged, so toff may go out of scope
      cudaError_t e = cudaMemcpyAsync(dtoff, toff.data(), sizeof(long long) * (nmol + 1),
                                      cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) {
        k_grad_xc<<<(unsigned)toff[nmol], B2G_XC_THREADS, smem, st>>>(P.mols, nmol, P.shells, P.g.grid_off,
                                                                       dtoff, coords, weights, D, grad);
        b2_count_launches(1);
        e = cudaGetLastError();
      }
      b2_dfree(dtoff, st);
      if (e != cudaSuccess) return B2_ERR_CUDA;
    }
  }
  if (parts & 8) {
    k_grad_nuc<<<nmol, 128, 0, st>>>(P.mols, P.atom_xyz, P.atom_z, grad);
    b2_count_launches(1);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
