// Exchange-correlation grid path (sm_100a), SIMT form.
//
// Replaces ``mol.eval_gto('GTOval_sph_deriv1', coords, 4)`` (dft.py:220) and the
// reference's ``exchange_correlation`` (nanoDFT.py:105-123, dft.py:899-1036):
//   rho_c[g] = sum_n (AO0 D)[g,n] AO_c[g,n]        c = 0..3  (rho_1..3 = half gradient)
//   (e_xc, vrho, vgamma) = B3LYP(rho)                fused per point
//   E_xc = sum_g rho_0 w e_xc
//   rt = [vrho/2, 4 vgamma rho_1..3] * w
//   V_xc = AO0^T (sum_c AO_c * rt_c),  V_xc <- V_xc + V_xc^T
// AO values are stored per molecule as [4][G][nao] (component-major, grid rows).
#include "device_plan.cuh"
#include "devmem.cuh"
#include "xc_math.cuh"
#include "xc.cuh"

// block index -> molecule via prefix over ceil(G/bs)
__device__ __forceinline__ int b2_find(const long long *off, int n, long long x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename T>
__global__ void __launch_bounds__(128)
k_ao_eval(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
          const long long *__restrict__ gblk_off, const long long *__restrict__ grid_off,
          const long long *__restrict__ ao_off, int nmol, const double *__restrict__ coords,
          T *__restrict__ ao) {
  const int m = b2_find(gblk_off, nmol, blockIdx.x);
  const B2MolDev md = mols[m];
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long g = (blockIdx.x - gblk_off[m]) * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const double *rc = coords + 3 * (grid_off[m] + g);
  const double x = rc[0], y = rc[1], z = rc[2];
  const int N = md.nao;
  T *a0 = ao + ao_off[m] + g * N;
  const long long cs = G * N;                 // component stride
  for (int s = 0; s < md.nbas; ++s) {
    const B2Shell sh = shells[md.sh_off + s];
    const double dx = x - sh.R[0], dy = y - sh.R[1], dz = z - sh.R[2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    double g0 = 0, g1 = 0;
    for (int k = 0; k < sh.nprim; ++k) {
      const double e = sh.coef[k] * exp(-sh.exp[k] * r2);
      g0 += e;
      g1 += -2.0 * sh.exp[k] * e;
    }
    if (sh.l == 0) {
      a0[sh.ao0] = (T)g0;
      a0[cs + sh.ao0] = (T)(g1 * dx);
      a0[2 * cs + sh.ao0] = (T)(g1 * dy);
      a0[3 * cs + sh.ao0] = (T)(g1 * dz);
    } else {
      const double d[3] = {dx, dy, dz};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        a0[sh.ao0 + c] = (T)(d[c] * g0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
          a0[(k + 1) * cs + sh.ao0 + c] = (T)((c == k ? g0 : 0.0) + d[c] * d[k] * g1);
      }
    }
  }
}

// Fused XC tile kernel: a CTA owns TPC consecutive tiles of PT points of one molecule.
// Per tile: the 4 AO components (PT x nao) are staged in shared memory; threads (tx, ty) of a
// 16x16 layout compute X = AO0 * D register-blocked (points ty+16r, orbitals tx+16q), reduce
// rho_c = sum_n X AO_c across the 16 tx lanes with shuffles, evaluate B3LYP per point, form
// Y = sum_c AO_c rt_c in place and accumulate V += AO0^T Y in registers (rows ty+16r, cols
// tx+16q) across the CTA's tiles; one float64 atomic flush per CTA.
#define B2_XC_NP 80          // padded orbital dimension (5 x 16)
template <typename T, int PT>
__global__ void __launch_bounds__(256)
k_xc_fused(const B2MolDev *__restrict__ mols, const long long *__restrict__ xblk_off,
           const long long *__restrict__ grid_off, const long long *__restrict__ ao_off, int nmol,
           int tpc, const int *__restrict__ active, const T *__restrict__ ao,
           const double *__restrict__ w, const double *__restrict__ D, double *__restrict__ V,
           double *__restrict__ exc) {
  constexpr int R = PT / 16;                 // points per thread (rows)
  constexpr int NP = B2_XC_NP, LD = NP + 1;  // odd leading dimension
  extern __shared__ unsigned char smem_raw[];
  T *sD = reinterpret_cast<T *>(smem_raw);             // [NP][NP]
  T *sA = sD + NP * NP;                                 // [4][PT][LD]
  __shared__ T sRt[PT][4];
  __shared__ double red[8];
  const int m = b2_find(xblk_off, nmol, blockIdx.x);
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  const int N = md.nao;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) {
    const int a = e / NP, b = e - (e / NP) * NP;
    sD[e] = (a < N && b < N) ? (T)D[md.mat_off + a * N + b] : (T)0;
  }
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long cs = G * N;
  const T *Am = ao + ao_off[m];
  const double *wm = w + grid_off[m];
  T vacc[5][5];
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int q = 0; q < 5; ++q) vacc[r][q] = (T)0;
  double e_part = 0;
  const long long t0 = (blockIdx.x - xblk_off[m]) * (long long)tpc;
  for (int tt = 0; tt < tpc; ++tt) {
    const long long g0 = (t0 + tt) * PT;
    if (g0 >= G) break;
    const int np = (int)min((long long)PT, G - g0);
    __syncthreads();                       // previous tile fully consumed
    for (int c = 0; c < 4; ++c) {
      const T *src = Am + c * cs + g0 * N;
      for (int e = threadIdx.x; e < PT * NP; e += blockDim.x) {
        const int p = e / NP, n = e - (e / NP) * NP;
        sA[(c * PT + p) * LD + n] = (p < np && n < N) ? src[p * N + n] : (T)0;
      }
    }
    __syncthreads();
    // X = AO0 * D
    T x[R][5];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) x[r][q] = (T)0;
    for (int k = 0; k < N; ++k) {
      T a[R], d[5];
#pragma unroll
      for (int r = 0; r < R; ++r) a[r] = sA[(ty + 16 * r) * LD + k];
#pragma unroll
      for (int q = 0; q < 5; ++q) d[q] = sD[k * NP + tx + 16 * q];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) x[r][q] += a[r] * d[q];
    }
    // rho_c for the thread's points, reduced over the 16 tx lanes
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int p = ty + 16 * r;
      T rc[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        T s = 0;
#pragma unroll
        for (int q = 0; q < 5; ++q) s += x[r][q] * sA[(c * PT + p) * LD + tx + 16 * q];
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        rc[c] = s;
      }
      if (tx == 0) {
        double wg = 0;
        T rt0 = 0, f4 = 0;
        if (p < np) {
          const B2XcPoint<T> o = b2_b3lyp_point<T>(rc[0], rc[1], rc[2], rc[3]);
          wg = wm[g0 + p];
          e_part += (double)rc[0] * wg * (double)o.exc;
          rt0 = o.vrho * (T)0.5 * (T)wg;
          f4 = (T)4 * o.vgamma * (T)wg;
        }
        sRt[p][0] = rt0;
        sRt[p][1] = f4 * rc[1];
        sRt[p][2] = f4 * rc[2];
        sRt[p][3] = f4 * rc[3];
      }
    }
    __syncthreads();
    // Y = sum_c AO_c rt_c (into the AO_x tile)
    for (int e = threadIdx.x; e < PT * NP; e += blockDim.x) {
      const int p = e / NP, n = e - (e / NP) * NP;
      const T y = sA[p * LD + n] * sRt[p][0] + sA[(PT + p) * LD + n] * sRt[p][1] +
                  sA[(2 * PT + p) * LD + n] * sRt[p][2] + sA[(3 * PT + p) * LD + n] * sRt[p][3];
      sA[(PT + p) * LD + n] = y;
    }
    __syncthreads();
    // V += AO0^T Y
    for (int p = 0; p < np; ++p) {
      T a[5], y[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) a[r] = sA[p * LD + ty + 16 * r];
#pragma unroll
      for (int q = 0; q < 5; ++q) y[q] = sA[(PT + p) * LD + tx + 16 * q];
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) vacc[r][q] += a[r] * y[q];
    }
  }
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int a = ty + 16 * r, b = tx + 16 * q;
      if (a < N && b < N && vacc[r][q] != (T)0) atomicAdd(&V[md.mat_off + a * N + b], (double)vacc[r][q]);
    }
  for (int o = 16; o > 0; o >>= 1) e_part += __shfl_down_sync(0xffffffffu, e_part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e_part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < 8; ++i) s += red[i];
    atomicAdd(&exc[m], s);
  }
}

// V <- V + V^T per molecule
__global__ void k_sym(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
                      double *__restrict__ V) {
  if (active && !active[blockIdx.x]) return;
  const B2MolDev md = mols[blockIdx.x];
  const int N = md.nao;
  double *v = V + md.mat_off;
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    if (a < b) {
      const double s = v[a * N + b] + v[b * N + a];
      v[a * N + b] = s;
      v[b * N + a] = s;
    } else if (a == b) {
      v[e] *= 2.0;
    }
  }
}

static void b2_xc_split(const std::vector<long long> &goff, int nmol, int pt, int &tpc,
                        std::vector<long long> &xblk, int tpc_fixed = 0) {
  long long tiles = 0;
  for (int m = 0; m < nmol; ++m) tiles += (goff[m + 1] - goff[m] + pt - 1) / pt;
  // enough CTAs to fill the GPU several times over, each flushing V once
  tpc = tpc_fixed > 0 ? tpc_fixed : (int)std::max(1ll, std::min(16ll, tiles / (8ll * 148ll)));
  xblk.assign(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    const long long nt = (goff[m + 1] - goff[m] + pt - 1) / pt;
    xblk[m + 1] = xblk[m] + (nt + tpc - 1) / tpc;
  }
}

int b2_grid_setup(B2PlanDev &P, const long long *grid_off_host) {
  b2_grid_free(P);
  const int nmol = P.h.nmol;
  std::vector<long long> goff(grid_off_host, grid_off_host + nmol + 1), gblk(nmol + 1, 0),
      aoff(nmol + 1, 0), x32, x64, xtc;
  for (int m = 0; m < nmol; ++m) {
    long long G = goff[m + 1] - goff[m];
    if (G < 0) return B2_ERR_ARG;
    gblk[m + 1] = gblk[m] + (G + 127) / 128;
    aoff[m + 1] = aoff[m] + 4 * G * P.h.mols[m].nao;
  }
  b2_xc_split(goff, nmol, 64, P.g.tpc32, x32);
  b2_xc_split(goff, nmol, 32, P.g.tpc64, x64);
  b2_xc_split(goff, nmol, 128, P.g.tpc_tc, xtc);
  P.g.n_points = goff[nmol];
  P.g.n_gblk = gblk[nmol];
  P.g.n_xblk32 = x32[nmol];
  P.g.n_xblk64 = x64[nmol];
  P.g.n_xblk_tc = xtc[nmol];
  P.g.n_ao = aoff[nmol];
  P.g.grid_off_h = goff;
  P.g.ao_off_h = aoff;
  P.g.xblk32_h = x32;
  P.g.xblk64_h = x64;
  P.g.xblk_tc_h = xtc;
  size_t nb = sizeof(long long) * (nmol + 1);
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.grid_off, nb));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.gblk_off, nb));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.xblk32, nb));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.xblk64, nb));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.xblk_tc, nb));
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.ao_off, nb));
  B2_CUDA_TRY(cudaMemcpy(P.g.grid_off, goff.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.gblk_off, gblk.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.xblk32, x32.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.xblk64, x64.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.xblk_tc, xtc.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.ao_off, aoff.data(), nb, cudaMemcpyHostToDevice));
  std::vector<int> all(nmol);
  for (int m = 0; m < nmol; ++m) all[m] = m;
  int rc = b2_xq_build(P, all, &P.g.xq_items, P.g.xq_off_h);
  if (rc) return rc;
  B2_CUDA_TRY(b2_dmalloc_t(&P.g.xq_queue, sizeof(int) * B2_NBKT));
  return B2_OK;
}

int b2_xc_set_tpc(B2PlanDev &P, int tpc) {
  if (!P.g.grid_off || tpc < 0) return B2_ERR_ARG;
  for (int b = 0; b < B2_NBKT; ++b) P.g.xq_tpc[b] = 0;    // one value for every bucket
  std::vector<long long> xtc;
  b2_xc_split(P.g.grid_off_h, P.h.nmol, 128, P.g.tpc_tc, xtc, tpc);
  long long *d = nullptr;
  const size_t nb = sizeof(long long) * (P.h.nmol + 1);
  B2_CUDA_TRY(b2_dmalloc_t(&d, nb));
  B2_CUDA_TRY(cudaMemcpy(d, xtc.data(), nb, cudaMemcpyHostToDevice));
  b2_dfree(P.g.xblk_tc);
  P.g.xblk_tc = d;
  P.g.xblk_tc_h = xtc;
  P.g.n_xblk_tc = xtc[P.h.nmol];
  std::vector<int> all(P.h.nmol);
  for (int m = 0; m < P.h.nmol; ++m) all[m] = m;
  return b2_xq_build(P, all, &P.g.xq_items, P.g.xq_off_h);
}

void b2_grid_free(B2PlanDev &P) {
  b2_dfree(P.g.grid_off); b2_dfree(P.g.gblk_off); b2_dfree(P.g.xblk32); b2_dfree(P.g.xblk64);
  b2_dfree(P.g.xblk_tc);
  b2_dfree(P.g.ao_off);
  b2_dfree(P.g.tmpl); b2_dfree(P.g.tmpl_off); b2_dfree(P.g.atom_pt_off);
  b2_dfree(P.g.xq_items); b2_dfree(P.g.xq_queue);
  P.g = B2GridDev();
}

int b2_launch_ao_eval(const B2PlanDev &P, int precision, const double *coords, void *ao,
                      cudaStream_t st) {
  if (!P.g.grid_off) return B2_ERR_ARG;
  if (P.g.n_gblk == 0) return B2_OK;
  if (precision == 64)
    k_ao_eval<double><<<(unsigned)P.g.n_gblk, 128, 0, st>>>(P.mols, P.shells, P.g.gblk_off,
        P.g.grid_off, P.g.ao_off, P.h.nmol, coords, (double *)ao);
  else if (precision == 32)
    k_ao_eval<float><<<(unsigned)P.g.n_gblk, 128, 0, st>>>(P.mols, P.shells, P.g.gblk_off,
        P.g.grid_off, P.g.ao_off, P.h.nmol, coords, (float *)ao);
  else return B2_ERR_ARG;
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

__global__ void k_zero_exc(int nmol, const int *__restrict__ active, double *__restrict__ exc) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nmol && (!active || active[m])) exc[m] = 0.0;
}

template <typename T, int PT>
static int b2_xc_impl(const B2PlanDev &P, const int *active, const T *ao, const double *w,
                      const double *D, double *V, double *exc, const long long *xblk, long long nblk,
                      int tpc, cudaStream_t st) {
  if (active) {
    int rc = b2_zero_active(P, active, V, nullptr, st);
    if (rc) return rc;
  } else {
    B2_CUDA_TRY(cudaMemsetAsync(V, 0, sizeof(double) * P.h.n_mat, st));
  }
  k_zero_exc<<<(P.h.nmol + 255) / 256, 256, 0, st>>>(P.h.nmol, active, exc);
  b2_count_launches(1);
  const size_t sm = sizeof(T) * (B2_XC_NP * B2_XC_NP + 4 * PT * (B2_XC_NP + 1));
  B2_CUDA_TRY(cudaFuncSetAttribute(k_xc_fused<T, PT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  if (nblk > 0) {
    k_xc_fused<T, PT><<<(unsigned)nblk, 256, sm, st>>>(P.mols, xblk, P.g.grid_off, P.g.ao_off,
                                                       P.h.nmol, tpc, active, ao, w, D, V, exc);
    b2_count_launches(1);
  }
  k_sym<<<P.h.nmol, 256, 0, st>>>(P.mols, active, V);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_xc(const B2PlanDev &P, int precision, const int *active, const void *ao,
                 const double *w, const double *D, double *V, double *exc, cudaStream_t st) {
  if (!P.g.grid_off) return B2_ERR_ARG;
  if (precision == 64)
    return b2_xc_impl<double, 32>(P, active, (const double *)ao, w, D, V, exc, P.g.xblk64,
                                  P.g.n_xblk64, P.g.tpc64, st);
  if (precision == 32)
    return b2_xc_impl<float, 64>(P, active, (const float *)ao, w, D, V, exc, P.g.xblk32,
                                 P.g.n_xblk32, P.g.tpc32, st);
  return B2_ERR_ARG;
}
