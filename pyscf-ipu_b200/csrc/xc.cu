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

// rho + B3LYP per point; writes rt[4][G] (scratch) and accumulates E_xc per molecule
template <typename T>
__global__ void __launch_bounds__(128)
k_rho_b3lyp(const B2MolDev *__restrict__ mols, const long long *__restrict__ gblk_off,
            const long long *__restrict__ grid_off, const long long *__restrict__ ao_off, int nmol,
            const T *__restrict__ ao, const double *__restrict__ w, const double *__restrict__ D,
            T *__restrict__ rt, double *__restrict__ exc) {
  __shared__ T sD[B2_MAXNAO * B2_MAXNAO];
  __shared__ double red[4];
  const int m = b2_find(gblk_off, nmol, blockIdx.x);
  const B2MolDev md = mols[m];
  const int N = md.nao;
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) sD[e] = (T)D[md.mat_off + e];
  __syncthreads();
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long g = (blockIdx.x - gblk_off[m]) * blockDim.x + threadIdx.x;
  double e_part = 0;
  if (g < G) {
    const long long cs = G * N;
    const T *a0 = ao + ao_off[m] + g * N;
    T r0 = 0, r1 = 0, r2 = 0, r3 = 0;
    for (int n = 0; n < N; ++n) {
      T xn = 0;
      for (int k = 0; k < N; ++k) xn += a0[k] * sD[k * N + n];
      r0 += xn * a0[n];
      r1 += xn * a0[cs + n];
      r2 += xn * a0[2 * cs + n];
      r3 += xn * a0[3 * cs + n];
    }
    const B2XcPoint<T> o = b2_b3lyp_point<T>(r0, r1, r2, r3);
    const double wg = w[grid_off[m] + g];
    e_part = (double)r0 * wg * (double)o.exc;
    T *rtm = rt + 4 * grid_off[m];
    rtm[g] = (T)(o.vrho * (T)0.5 * (T)wg);
    const T f4 = (T)4 * o.vgamma * (T)wg;
    rtm[G + g] = f4 * r1;
    rtm[2 * G + g] = f4 * r2;
    rtm[3 * G + g] = f4 * r3;
  }
  // block reduction of e_part
  for (int o = 16; o > 0; o >>= 1) e_part += __shfl_down_sync(0xffffffffu, e_part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e_part;
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(&exc[m], red[0] + red[1] + red[2] + red[3]);
}

// V_raw[a,b] += sum_g AO0[g,a] * (sum_c AO_c[g,b] rt_c[g]) over a chunk of points
#define B2_VXC_PTS 64
template <typename T>
__global__ void __launch_bounds__(256)
k_vxc(const B2MolDev *__restrict__ mols, const long long *__restrict__ vblk_off,
      const long long *__restrict__ grid_off, const long long *__restrict__ ao_off, int nmol,
      const T *__restrict__ ao, const T *__restrict__ rt, double *__restrict__ V) {
  extern __shared__ unsigned char smem_raw[];
  T *sA = reinterpret_cast<T *>(smem_raw);                 // [PTS][N]
  const int m = b2_find(vblk_off, nmol, blockIdx.x);
  const B2MolDev md = mols[m];
  const int N = md.nao;
  T *sY = sA + B2_VXC_PTS * N;                            // [PTS][N]
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long g0 = (blockIdx.x - vblk_off[m]) * B2_VXC_PTS;
  const int np = (int)min((long long)B2_VXC_PTS, G - g0);
  const long long cs = G * N;
  const T *A = ao + ao_off[m];
  const T *R = rt + 4 * grid_off[m];
  for (int e = threadIdx.x; e < np * N; e += blockDim.x) {
    const int p = e / N, b = e - (e / N) * N;
    const long long gi = g0 + p;
    sA[p * N + b] = A[gi * N + b];
    sY[p * N + b] = A[gi * N + b] * R[gi] + A[cs + gi * N + b] * R[G + gi] +
                    A[2 * cs + gi * N + b] * R[2 * G + gi] + A[3 * cs + gi * N + b] * R[3 * G + gi];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    T s = 0;
    for (int p = 0; p < np; ++p) s += sA[p * N + a] * sY[p * N + b];
    atomicAdd(&V[md.mat_off + e], (double)s);
  }
}

// V <- V + V^T per molecule
__global__ void k_sym(const B2MolDev *__restrict__ mols, double *__restrict__ V) {
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

int b2_grid_setup(B2PlanDev &P, const long long *grid_off_host) {
  b2_grid_free(P);
  const int nmol = P.h.nmol;
  std::vector<long long> goff(grid_off_host, grid_off_host + nmol + 1), gblk(nmol + 1, 0),
      vblk(nmol + 1, 0), aoff(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    long long G = goff[m + 1] - goff[m];
    if (G < 0) return B2_ERR_ARG;
    gblk[m + 1] = gblk[m] + (G + 127) / 128;
    vblk[m + 1] = vblk[m] + (G + B2_VXC_PTS - 1) / B2_VXC_PTS;
    aoff[m + 1] = aoff[m] + 4 * G * P.h.mols[m].nao;
  }
  P.g.n_points = goff[nmol];
  P.g.n_gblk = gblk[nmol];
  P.g.n_vblk = vblk[nmol];
  P.g.n_ao = aoff[nmol];
  P.g.grid_off_h = goff;
  P.g.ao_off_h = aoff;
  size_t nb = sizeof(long long) * (nmol + 1);
  B2_CUDA_TRY(cudaMalloc(&P.g.grid_off, nb));
  B2_CUDA_TRY(cudaMalloc(&P.g.gblk_off, nb));
  B2_CUDA_TRY(cudaMalloc(&P.g.vblk_off, nb));
  B2_CUDA_TRY(cudaMalloc(&P.g.ao_off, nb));
  B2_CUDA_TRY(cudaMemcpy(P.g.grid_off, goff.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.gblk_off, gblk.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.vblk_off, vblk.data(), nb, cudaMemcpyHostToDevice));
  B2_CUDA_TRY(cudaMemcpy(P.g.ao_off, aoff.data(), nb, cudaMemcpyHostToDevice));
  // scratch for rt (4 x points) in double (covers both precisions)
  B2_CUDA_TRY(cudaMalloc(&P.g.rt, sizeof(double) * 4 * std::max<long long>(1, P.g.n_points)));
  return B2_OK;
}

void b2_grid_free(B2PlanDev &P) {
  cudaFree(P.g.grid_off); cudaFree(P.g.gblk_off); cudaFree(P.g.vblk_off); cudaFree(P.g.ao_off);
  cudaFree(P.g.rt);
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
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

template <typename T>
static int b2_xc_impl(const B2PlanDev &P, const T *ao, const double *w, const double *D, double *V,
                      double *exc, T *rt, cudaStream_t st) {
  B2_CUDA_TRY(cudaMemsetAsync(V, 0, sizeof(double) * P.h.n_mat, st));
  B2_CUDA_TRY(cudaMemsetAsync(exc, 0, sizeof(double) * P.h.nmol, st));
  if (P.g.n_gblk > 0)
    k_rho_b3lyp<T><<<(unsigned)P.g.n_gblk, 128, 0, st>>>(P.mols, P.g.gblk_off, P.g.grid_off,
        P.g.ao_off, P.h.nmol, ao, w, D, rt, exc);
  const int N = P.h.max_nao;
  size_t sm = sizeof(T) * 2 * B2_VXC_PTS * N;
  B2_CUDA_TRY(cudaFuncSetAttribute(k_vxc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  if (P.g.n_vblk > 0)
    k_vxc<T><<<(unsigned)P.g.n_vblk, 256, sm, st>>>(P.mols, P.g.vblk_off, P.g.grid_off, P.g.ao_off,
                                                    P.h.nmol, ao, rt, V);
  k_sym<<<P.h.nmol, 256, 0, st>>>(P.mols, V);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_xc(const B2PlanDev &P, int precision, const void *ao, const double *w,
                 const double *D, double *V, double *exc, void *rt_scratch, cudaStream_t st) {
  if (!P.g.grid_off) return B2_ERR_ARG;
  if (precision == 64)
    return b2_xc_impl<double>(P, (const double *)ao, w, D, V, exc, (double *)rt_scratch, st);
  if (precision == 32)
    return b2_xc_impl<float>(P, (const float *)ao, w, D, V, exc, (float *)rt_scratch, st);
  return B2_ERR_ARG;
}
