// Per-molecule setup on the device (sm_100a): one-electron matrices, Becke grid, guess,
// nuclear repulsion.  These replace the host PySCF calls of the reference
// (int1e_ovlp/kin/nuc dft.py:225-227, Grids.build dft.py:214-216 / build_grid.py:109-135,
// minao dft.py:223, energy_nuc dft.py:202) and follow the same formulas as the package's
// host versions (b200dft/int1e.py, b200dft/grids.py, b200dft/guess.py), so the device
// setup reproduces the host setup to rounding.
#include <algorithm>
#include <vector>
#include "device_plan.cuh"
#include "devmem.cuh"
#include "setup.cuh"

// ------------------------------------------------------------------ one-electron matrices
// Every s/p primitive is d.(r-P) + s times the Gaussian product at P (d = 0, s = 1 for s):
//   overlap  <fa fb> = sa sb + (da.db) u,                           u = 1/(2 zeta)
//   r_B^2    <fa fb |r-B|^2> = sa sb |PB|^2 + u[(da.db)|PB|^2 + 2 sb da.PB + 2 sa db.PB + 3 sa sb]
//                              + 5 u^2 (da.db)
//   kinetic  T = -1/2 [4 b^2 <r_B^2> - 2 b (3 + 2 l_b) <1>]
//   nuclear  V = sum_C -Z_C (2 pi / zeta) K [E0 f0 + u (sb Xa + sa Xb) f1 + u^2 (da.db f1 + Xa Xb f2)]
__global__ void __launch_bounds__(256)
k_int1e(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
        const int *__restrict__ ao2sh, const double *__restrict__ atom_xyz,
        const int *__restrict__ atom_z, const double *__restrict__ btab, double *__restrict__ S,
        double *__restrict__ T, double *__restrict__ V) {
  const B2MolDev md = mols[blockIdx.x];
  const int N = md.nao;
  const int npair = N * (N + 1) / 2;
  for (int pidx = threadIdx.x; pidx < npair; pidx += blockDim.x) {
    const int a = (int)b2_untri(pidx);
    const int b = pidx - a * (a + 1) / 2;
    const B2Shell A = shells[md.sh_off + ao2sh[md.ao_off + a]];
    const B2Shell B = shells[md.sh_off + ao2sh[md.ao_off + b]];
    double da[3] = {0, 0, 0}, db[3] = {0, 0, 0};
    if (A.l) da[a - A.ao0] = 1.0;
    if (B.l) db[b - B.ao0] = 1.0;
    const double dab = da[0] * db[0] + da[1] * db[1] + da[2] * db[2];
    double AB2 = 0;
    for (int d = 0; d < 3; ++d) AB2 += (A.R[d] - B.R[d]) * (A.R[d] - B.R[d]);
    double s_acc = 0, t_acc = 0, v_acc = 0;
    for (int pa = 0; pa < A.nprim; ++pa)
      for (int pb = 0; pb < B.nprim; ++pb) {
        const double al = A.exp[pa], be = B.exp[pb], z = al + be, u = 0.5 / z;
        const double cc = A.coef[pa] * B.coef[pb];
        const double K = exp(-al * be / z * AB2);
        double P[3], PA[3], PB[3];
        for (int d = 0; d < 3; ++d) {
          P[d] = (al * A.R[d] + be * B.R[d]) / z;
          PA[d] = P[d] - A.R[d];
          PB[d] = P[d] - B.R[d];
        }
        const double sa = A.l ? da[0] * PA[0] + da[1] * PA[1] + da[2] * PA[2] : 1.0;
        const double sb = B.l ? db[0] * PB[0] + db[1] * PB[1] + db[2] * PB[2] : 1.0;
        const double sprim = pow(M_PI / z, 1.5) * K;
        const double ov = sa * sb + dab * u;
        const double PB2 = PB[0] * PB[0] + PB[1] * PB[1] + PB[2] * PB[2];
        const double daPB = da[0] * PB[0] + da[1] * PB[1] + da[2] * PB[2];
        const double dbPB = db[0] * PB[0] + db[1] * PB[1] + db[2] * PB[2];
        const double r2 = sa * sb * PB2 + u * (dab * PB2 + 2 * sb * daPB + 2 * sa * dbPB + 3 * sa * sb) +
                          5 * u * u * dab;
        s_acc += cc * sprim * ov;
        t_acc += cc * sprim * (-0.5) * (4 * be * be * r2 - 2 * be * (3 + 2 * B.l) * ov);
        const double E0 = sa * sb + dab * u;
        double vsum = 0;
        for (int c = 0; c < md.natm; ++c) {
          const double *C = atom_xyz + 3 * (md.atm_off + c);
          const double X[3] = {P[0] - C[0], P[1] - C[1], P[2] - C[2]};
          const double tt = z * (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
          double F[3];
          b2_boys<double, 2>(tt, btab, F);
          const double f0 = F[0], f1 = -2 * z * F[1], f2 = 4 * z * z * F[2];
          const double Xa = da[0] * X[0] + da[1] * X[1] + da[2] * X[2];
          const double Xb = db[0] * X[0] + db[1] * X[1] + db[2] * X[2];
          const double val = E0 * f0 + u * (sb * Xa + sa * Xb) * f1 + u * u * (dab * f1 + Xa * Xb * f2);
          vsum += -(double)atom_z[md.atm_off + c] * val;
        }
        v_acc += cc * (2 * M_PI / z) * K * vsum;
      }
    const long long o = md.mat_off;
    S[o + a * N + b] = s_acc; S[o + b * N + a] = s_acc;
    T[o + a * N + b] = t_acc; T[o + b * N + a] = t_acc;
    V[o + a * N + b] = v_acc; V[o + b * N + a] = v_acc;
  }
}

// ------------------------------------------------------------------ Becke grid
__constant__ double c_bragg_sqrt[10];     // sqrt of Bragg-Slater radius (Angstrom), by Z

__device__ __forceinline__ int b2_find_ll(const long long *off, int lo, int hi, long long x) {
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// One CTA per block of 128 grid points of one molecule, one thread per point: coordinate from
// the owning atom's template, weight = template weight * Becke cell function (3-fold
// polynomial, size-adjusted, build_grid.py:34-100) normalised over atoms.  The CTA tabulates
// 1/R_ij and the size adjustments a_ij of its molecule in shared memory; each unordered atom
// pair is evaluated once per point, using a_ji = -a_ij and the odd polynomial, so
// s(nu_ji) = 1 - s(nu_ij).  Per-point distances and cell products live in shared memory.
#define B2_GRID_MAXATM 32
__global__ void __launch_bounds__(128)
k_grid(const B2MolDev *__restrict__ mols, int nmol, const long long *__restrict__ gblk_off,
       const long long *__restrict__ grid_off, const long long *__restrict__ atom_pt_off,
       const double *__restrict__ atom_xyz, const int *__restrict__ atom_z,
       const double *__restrict__ tmpl, const long long *__restrict__ tmpl_off,
       double *__restrict__ coords, double *__restrict__ weights) {
  __shared__ double sA[B2_GRID_MAXATM][3];
  extern __shared__ double sgrid[];                 // [na*na] 1/R, [na*na] a, [na][128] d, p
  const int m = b2_find_ll(gblk_off, 0, nmol - 1, blockIdx.x);
  const B2MolDev md = mols[m];
  const int na = md.natm, tid = threadIdx.x;
  double *sInv = sgrid, *sAij = sInv + na * na;
  double (*sDist)[128] = reinterpret_cast<double (*)[128]>(sAij + na * na);
  double (*sP)[128] = sDist + na;
  for (int e = tid; e < na; e += blockDim.x) {
    sA[e][0] = atom_xyz[3 * (md.atm_off + e)];
    sA[e][1] = atom_xyz[3 * (md.atm_off + e) + 1];
    sA[e][2] = atom_xyz[3 * (md.atm_off + e) + 2];
  }
  __syncthreads();
  for (int e = tid; e < na * na; e += blockDim.x) {
    const int i = e / na, j = e - (e / na) * na;
    double inv = 0.0, a = 0.0;
    if (i != j) {
      const double rx = sA[i][0] - sA[j][0], ry = sA[i][1] - sA[j][1], rz = sA[i][2] - sA[j][2];
      inv = 1.0 / sqrt(rx * rx + ry * ry + rz * rz);
      const double chi = c_bragg_sqrt[atom_z[md.atm_off + i]] / c_bragg_sqrt[atom_z[md.atm_off + j]];
      const double uu = (chi - 1) / (chi + 1);
      a = fmin(0.5, fmax(-0.5, uu / (uu * uu - 1)));
    }
    sInv[e] = inv;
    sAij[e] = a;
  }
  __syncthreads();
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long lp = (blockIdx.x - gblk_off[m]) * 128 + tid;    // point index in the molecule
  if (lp >= G) return;
  const long long gp = grid_off[m] + lp;
  const int ia = b2_find_ll(atom_pt_off, md.atm_off, md.atm_off + na - 1, gp) - md.atm_off;
  const int z = atom_z[md.atm_off + ia];
  const long long t = tmpl_off[z] + (gp - atom_pt_off[md.atm_off + ia]);
  const double x = sA[ia][0] + tmpl[4 * t], y = sA[ia][1] + tmpl[4 * t + 1], zc = sA[ia][2] + tmpl[4 * t + 2];
  coords[3 * gp] = x; coords[3 * gp + 1] = y; coords[3 * gp + 2] = zc;
  for (int i = 0; i < na; ++i) {
    const double dx = x - sA[i][0], dy = y - sA[i][1], dz = zc - sA[i][2];
    sDist[i][tid] = sqrt(dx * dx + dy * dy + dz * dz);
    sP[i][tid] = 1.0;
  }
  for (int i = 0; i < na; ++i) {
    const double di = sDist[i][tid];
    double pi = sP[i][tid];
    for (int j = i + 1; j < na; ++j) {
      const double mu = (di - sDist[j][tid]) * sInv[i * na + j];
      double g = mu + sAij[i * na + j] * (1 - mu * mu);
      g = (3 - g * g) * g * 0.5;
      g = (3 - g * g) * g * 0.5;
      g = (3 - g * g) * g * 0.5;
      pi *= 0.5 * (1 - g);
      sP[j][tid] *= 0.5 * (1 + g);
    }
    sP[i][tid] = pi;
  }
  double psum = 0;
  for (int i = 0; i < na; ++i) psum += sP[i][tid];
  weights[gp] = tmpl[4 * t + 3] * sP[ia][tid] / psum;
}

// ------------------------------------------------------------------ guess + E_nuc
// MINAO-style occupations on the diagonal: H 1s 1; heavy 1s 2, 2s 2, 2p (Z-4)/3 each
__global__ void k_guess(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
                        const int *__restrict__ ao2sh, const int *__restrict__ atom_z,
                        double *__restrict__ D) {
  const B2MolDev md = mols[blockIdx.x];
  const int N = md.nao;
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    double v = 0;
    if (a == b) {
      const int s = ao2sh[md.ao_off + a];
      const B2Shell sh = shells[md.sh_off + s];
      const int z = atom_z[md.atm_off + sh.atom];
      if (z <= 2) v = (double)z;
      else if (sh.l == 0) v = 2.0;
      else v = (z - 4) / 3.0;
    }
    D[md.mat_off + e] = v;
  }
}

__global__ void k_enuc(const B2MolDev *__restrict__ mols, int nmol, const double *__restrict__ atom_xyz,
                       const int *__restrict__ atom_z, double *__restrict__ enuc) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nmol) return;
  const B2MolDev md = mols[m];
  const double *A = atom_xyz + 3 * md.atm_off;
  double e = 0;
  for (int i = 0; i < md.natm; ++i)
    for (int j = 0; j < i; ++j) {
      const double dx = A[3 * i] - A[3 * j], dy = A[3 * i + 1] - A[3 * j + 1], dz = A[3 * i + 2] - A[3 * j + 2];
      e += (double)atom_z[md.atm_off + i] * atom_z[md.atm_off + j] / sqrt(dx * dx + dy * dy + dz * dz);
    }
  enuc[m] = e;
}

// s8 entries with |v| <= threshold become 0 (the ERI threshold of nanoDFT.py:280-288); the
// molecules' padding entries are never read, so the whole buffer is swept
template <typename T>
__global__ void k_threshold(long long n, T *__restrict__ x, double thr) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (fabs((double)x[i]) <= thr) x[i] = (T)0;
}

int b2_launch_eri_threshold(const B2PlanDev &P, int precision, void *eri, double thr, cudaStream_t st) {
  if (!eri || (precision != 32 && precision != 64) || !(thr >= 0.0)) return B2_ERR_ARG;
  const long long n = P.h.n_eri;
  if (n > 0) {
    const unsigned nb = (unsigned)std::min<long long>((n + 255) / 256, 148ll * 32);
    if (precision == 64) k_threshold<double><<<nb, 256, 0, st>>>(n, (double *)eri, thr);
    else k_threshold<float><<<nb, 256, 0, st>>>(n, (float *)eri, thr);
    b2_count_launches(1);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_int1e(const B2PlanDev &P, double *S, double *T, double *V, cudaStream_t st) {
  k_int1e<<<P.h.nmol, 256, 0, st>>>(P.mols, P.shells, P.ao2sh, P.atom_xyz, P.atom_z, P.boys, S, T, V);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_grid_build(B2PlanDev &P, int nz, const double *tmpl_host, const long long *tmpl_off_host,
                         double *coords, double *weights, cudaStream_t st) {
  if (!P.g.grid_off || nz < 10) return B2_ERR_ARG;
  for (int m = 0; m < P.h.nmol; ++m)
    if (P.h.mols[m].natm > 32) return B2_ERR_SIZE;      // per-point distance table in registers
  // per-atom point offsets from the templates; must agree with the registered grid layout
  std::vector<long long> apo(P.h.n_atm + 1, 0);
  long long tot = 0;
  for (int m = 0; m < P.h.nmol; ++m) {
    const B2MolDev &md = P.h.mols[m];
    if (tot != P.g.grid_off_h[m]) return B2_ERR_ARG;
    for (int a = 0; a < md.natm; ++a) {
      const int z = P.h.atom_z[md.atm_off + a];
      if (z < 0 || z >= nz) return B2_ERR_UNSUPPORTED;
      apo[md.atm_off + a] = tot;
      tot += tmpl_off_host[z + 1] - tmpl_off_host[z];
    }
  }
  apo[P.h.n_atm] = tot;
  if (tot != P.g.n_points) return B2_ERR_ARG;
  const long long ntm = tmpl_off_host[nz];
  b2_dfree(P.g.tmpl); b2_dfree(P.g.tmpl_off); b2_dfree(P.g.atom_pt_off);
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.tmpl, sizeof(double) * 4 * std::max(1ll, ntm)));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.tmpl_off, sizeof(long long) * (nz + 1)));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.atom_pt_off, sizeof(long long) * apo.size()));
  B2_CUDA_TRY(cudaMemcpy(P.g.tmpl, tmpl_host, sizeof(double) * 4 * ntm, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.tmpl_off, tmpl_off_host, sizeof(long long) * (nz + 1), cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.atom_pt_off, apo.data(), sizeof(long long) * apo.size(), cudaMemcpyHostToDevice));
  const double br[10] = {0.35, 0.35, 0, 0, 0, 0, 0.70, 0.65, 0.60, 0.50};
  double brs[10];
  for (int i = 0; i < 10; ++i) brs[i] = br[i] > 0 ? sqrt(br[i]) : 1.0;
  B2_CUDA_TRY(cudaMemcpyToSymbol(c_bragg_sqrt, brs, sizeof(brs)));
  if (P.g.n_points > 0) {
    if (P.h.max_natm > B2_GRID_MAXATM) return B2_ERR_SIZE;
    const size_t sm = sizeof(double) * (2 * P.h.max_natm * P.h.max_natm + 2 * 128 * P.h.max_natm);
    B2_CUDA_TRY(cudaFuncSetAttribute(k_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_grid<<<(unsigned)P.g.n_gblk, 128, sm, st>>>(P.mols, P.h.nmol, P.g.gblk_off, P.g.grid_off,
        P.g.atom_pt_off, P.atom_xyz, P.atom_z, P.g.tmpl, P.g.tmpl_off, coords, weights);
    b2_count_launches(1);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_guess(const B2PlanDev &P, double *D, cudaStream_t st) {
  k_guess<<<P.h.nmol, 256, 0, st>>>(P.mols, P.shells, P.ao2sh, P.atom_z, D);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_enuc(const B2PlanDev &P, double *enuc, cudaStream_t st) {
  k_enuc<<<(P.h.nmol + 127) / 128, 128, 0, st>>>(P.mols, P.h.nmol, P.atom_xyz, P.atom_z, enuc);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

