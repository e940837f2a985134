// Exchange-correlation without a stored AO tensor (sm_100a).
//
// Same result as b2_xc (exchange_correlation, nanoDFT.py:105-123) but the AO values and
// gradients of each tile of points are generated in shared memory from the basis (the
// reference evaluates them once on the host with eval_gto, dft.py:220, and streams the
// (4, G, N) tensor every iteration).  Per tile of PT points:
//   AO, dAO/dx,y,z  -> shared memory            (thread per (point, shell))
//   X = AO0 D       -> registers                (thread (tx,ty): points ty+16r, orbitals tx+16q)
//   rho_c = sum_n X AO_c                        (shuffle reduction over the 16 tx lanes)
//   B3LYP per point -> rt = [vrho/2, 4 vgamma rho_1..3] * w
//   Y = sum_c AO_c rt_c, V += AO0^T Y            (registers across the CTA's tiles)
// The orbital dimension is padded to the molecule's bucket NB = 16*Q (Q = 1..5), a
// compile-time choice per CTA, so small molecules do not pay for nao = 70.
#include "device_plan.cuh"
#include "xc_math.cuh"
#include "xc.cuh"

#define B2_XD_MAXSH 48

__device__ __forceinline__ int b2_findx(const long long *off, int n, long long x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename T, int PT, int Q>
__device__ __forceinline__ void b2_xd_body(const B2MolDev &md, const B2Shell *sh, T *sD, T *sA,
                                           T (*sRt)[4], double *sC, const double *__restrict__ coords,
                                           const double *__restrict__ w, long long G, long long t0,
                                           int tpc, double *__restrict__ V, double &e_part) {
  constexpr int R = PT / 16, NB = 16 * Q, LD = NB + 1;
  const int N = md.nao, nbas = md.nbas;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T vacc[Q][Q];
#pragma unroll
  for (int r = 0; r < Q; ++r)
#pragma unroll
    for (int q = 0; q < Q; ++q) vacc[r][q] = (T)0;
  for (int tt = 0; tt < tpc; ++tt) {
    const long long g0 = (t0 + tt) * PT;
    if (g0 >= G) break;
    const int np = (int)min((long long)PT, G - g0);
    __syncthreads();                                   // previous tile consumed
    for (int e = threadIdx.x; e < PT * 3; e += blockDim.x) {
      const int p = e / 3, d = e - (e / 3) * 3;
      sC[e] = (p < np) ? coords[3 * (g0 + p) + d] : 1e30;
    }
    for (int e = threadIdx.x; e < 4 * PT * NB; e += blockDim.x) {   // clear (pads stay zero)
      const int cp = e / NB, n = e - (e / NB) * NB;
      sA[cp * LD + n] = (T)0;
    }
    __syncthreads();
    // AO values + gradients
    for (int e = threadIdx.x; e < PT * nbas; e += blockDim.x) {
      const int p = e / nbas, s = e - (e / nbas) * nbas;
      if (p >= np) continue;
      const B2Shell &S = sh[s];
      const T dx = (T)(sC[3 * p] - S.R[0]), dy = (T)(sC[3 * p + 1] - S.R[1]), dz = (T)(sC[3 * p + 2] - S.R[2]);
      const T r2 = dx * dx + dy * dy + dz * dz;
      T ga = 0, gb = 0;
      for (int k = 0; k < S.nprim; ++k) {
        const T ax = (T)S.exp[k] * r2;
        if (ax > (T)60) continue;
        const T ev = (T)S.coef[k] * exp(-ax);
        ga += ev;
        gb += (T)(-2.0 * S.exp[k]) * ev;
      }
      if (S.l == 0) {
        sA[(0 * PT + p) * LD + S.ao0] = ga;
        sA[(1 * PT + p) * LD + S.ao0] = gb * dx;
        sA[(2 * PT + p) * LD + S.ao0] = gb * dy;
        sA[(3 * PT + p) * LD + S.ao0] = gb * dz;
      } else {
        const T dd[3] = {dx, dy, dz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sA[(0 * PT + p) * LD + S.ao0 + c] = dd[c] * ga;
#pragma unroll
          for (int k = 0; k < 3; ++k)
            sA[((1 + k) * PT + p) * LD + S.ao0 + c] = (c == k ? ga : (T)0) + dd[c] * dd[k] * gb;
        }
      }
    }
    __syncthreads();
    // X = AO0 * D
    T x[R][Q];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int q = 0; q < Q; ++q) x[r][q] = (T)0;
    for (int k = 0; k < N; ++k) {
      T a[R], d[Q];
#pragma unroll
      for (int r = 0; r < R; ++r) a[r] = sA[(ty + 16 * r) * LD + k];
#pragma unroll
      for (int q = 0; q < Q; ++q) d[q] = sD[k * NB + tx + 16 * q];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int q = 0; q < Q; ++q) x[r][q] += a[r] * d[q];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int p = ty + 16 * r;
      T rc[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        T s = 0;
#pragma unroll
        for (int q = 0; q < Q; ++q) s += x[r][q] * sA[(c * PT + p) * LD + tx + 16 * q];
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        rc[c] = s;
      }
      if (tx == 0) {
        T rt0 = 0, f4 = 0;
        if (p < np) {
          const B2XcPoint<T> o = b2_b3lyp_point<T>(rc[0], rc[1], rc[2], rc[3]);
          const double wg = w[g0 + p];
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
    for (int e = threadIdx.x; e < PT * NB; e += blockDim.x) {
      const int p = e / NB, n = e - (e / NB) * NB;
      sA[(PT + p) * LD + n] = sA[p * LD + n] * sRt[p][0] + sA[(PT + p) * LD + n] * sRt[p][1] +
                              sA[(2 * PT + p) * LD + n] * sRt[p][2] + sA[(3 * PT + p) * LD + n] * sRt[p][3];
    }
    __syncthreads();
    for (int p = 0; p < np; ++p) {
      T a[Q], y[Q];
#pragma unroll
      for (int r = 0; r < Q; ++r) a[r] = sA[p * LD + ty + 16 * r];
#pragma unroll
      for (int q = 0; q < Q; ++q) y[q] = sA[(PT + p) * LD + tx + 16 * q];
#pragma unroll
      for (int r = 0; r < Q; ++r)
#pragma unroll
        for (int q = 0; q < Q; ++q) vacc[r][q] += a[r] * y[q];
    }
  }
#pragma unroll
  for (int r = 0; r < Q; ++r)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int a = ty + 16 * r, b = tx + 16 * q;
      if (a < N && b < N && vacc[r][q] != (T)0) atomicAdd(&V[md.mat_off + a * N + b], (double)vacc[r][q]);
    }
}

template <typename T, int PT>
__global__ void __launch_bounds__(256)
k_xc_direct(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
            const long long *__restrict__ xblk_off, const long long *__restrict__ grid_off, int nmol,
            int tpc, const int *__restrict__ active, const double *__restrict__ coords,
            const double *__restrict__ w, const double *__restrict__ D, double *__restrict__ V,
            double *__restrict__ exc, const int *__restrict__ mol_map) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ B2Shell sh[B2_XD_MAXSH];
  __shared__ T sRt[PT][4];
  __shared__ double sC[PT * 3];
  __shared__ double red[8];
  const int lo = b2_findx(xblk_off, nmol, blockIdx.x);
  const int m = mol_map ? mol_map[lo] : lo;
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  const int N = md.nao;
  const int Q = (N + 15) / 16, NB = 16 * Q;
  T *sD = reinterpret_cast<T *>(smem_raw);                  // [NB][NB]
  T *sA = sD + NB * NB;                                      // [4][PT][NB+1]
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int a = e / NB, b = e - (e / NB) * NB;
    sD[e] = (a < N && b < N) ? (T)D[md.mat_off + a * N + b] : (T)0;
  }
  for (int s = threadIdx.x; s < md.nbas; s += blockDim.x) sh[s] = shells[md.sh_off + s];
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long t0 = (blockIdx.x - xblk_off[lo]) * (long long)tpc;
  const double *cm = coords + 3 * grid_off[m];
  const double *wm = w + grid_off[m];
  double e_part = 0;
  switch (Q) {
    case 1: b2_xd_body<T, PT, 1>(md, sh, sD, sA, sRt, sC, cm, wm, G, t0, tpc, V, e_part); break;
    case 2: b2_xd_body<T, PT, 2>(md, sh, sD, sA, sRt, sC, cm, wm, G, t0, tpc, V, e_part); break;
    case 3: b2_xd_body<T, PT, 3>(md, sh, sD, sA, sRt, sC, cm, wm, G, t0, tpc, V, e_part); break;
    case 4: b2_xd_body<T, PT, 4>(md, sh, sD, sA, sRt, sC, cm, wm, G, t0, tpc, V, e_part); break;
    default: b2_xd_body<T, PT, 5>(md, sh, sD, sA, sRt, sC, cm, wm, G, t0, tpc, V, e_part); break;
  }
  for (int o = 16; o > 0; o >>= 1) e_part += __shfl_down_sync(0xffffffffu, e_part, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e_part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < 8; ++i) s += red[i];
    atomicAdd(&exc[m], s);
  }
}

__global__ void k_zero_exc2(int nmol, const int *__restrict__ active, double *__restrict__ exc) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nmol && (!active || active[m])) exc[m] = 0.0;
}

__global__ void k_sym2(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
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

int b2_zero_exc(const B2PlanDev &P, const int *active, double *exc, cudaStream_t st) {
  k_zero_exc2<<<(P.h.nmol + 255) / 256, 256, 0, st>>>(P.h.nmol, active, exc);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_sym_v(const B2PlanDev &P, const int *active, double *V, cudaStream_t st) {
  k_sym2<<<P.h.nmol, 256, 0, st>>>(P.mols, active, V);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

template <typename T, int PT>
static int b2_xcd_impl(const B2PlanDev &P, const int *active, const double *coords, const double *w,
                       const double *D, double *V, double *exc, const long long *xblk,
                       long long nblk, int tpc, cudaStream_t st) {
  const bool sub = P.sub.n > 0;
  const int nm = sub ? P.sub.n : P.h.nmol;
  const int *map = sub ? P.sub.mol_map : nullptr;
  if (P.h.max_nbas > B2_XD_MAXSH) return B2_ERR_SIZE;
  if (active) {
    int rc = b2_zero_active(P, active, V, nullptr, st);
    if (rc) return rc;
  } else {
    B2_CUDA_TRY(cudaMemsetAsync(V, 0, sizeof(double) * P.h.n_mat, st));
  }
  k_zero_exc2<<<(P.h.nmol + 255) / 256, 256, 0, st>>>(P.h.nmol, active, exc);
  b2_count_launches(1);
  const int NBmax = 80;
  const size_t sm = sizeof(T) * (NBmax * NBmax + 4 * PT * (NBmax + 1));
  B2_CUDA_TRY(cudaFuncSetAttribute(k_xc_direct<T, PT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  if (nblk > 0) {
    k_xc_direct<T, PT><<<(unsigned)nblk, 256, sm, st>>>(P.mols, P.shells, xblk, P.g.grid_off, nm,
                                                         tpc, active, coords, w, D, V, exc, map);
    b2_count_launches(1);
  }
  k_sym2<<<P.h.nmol, 256, 0, st>>>(P.mols, active, V);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_xc_direct(const B2PlanDev &P, int precision, const int *active, const double *coords,
                        const double *w, const double *D, double *V, double *exc, cudaStream_t st) {
  if (!P.g.grid_off) return B2_ERR_ARG;
  const bool sub = P.sub.n > 0;
  if (precision == 64)
    return b2_xcd_impl<double, 32>(P, active, coords, w, D, V, exc, sub ? P.sub.x64 : P.g.xblk64,
                                   sub ? P.sub.n_x64 : P.g.n_xblk64, P.g.tpc64, st);
  if (precision == 32 && P.xc_impl == 0)
    return b2_launch_xc_tq(P, active, coords, w, D, V, exc, st);
  if (precision == 32 && P.xc_impl == 2)
    return b2_launch_xc_tc(P, active, coords, w, D, V, exc, st);
  if (precision == 32)
    return b2_xcd_impl<float, 64>(P, active, coords, w, D, V, exc, sub ? P.sub.x32 : P.g.xblk32,
                                  sub ? P.sub.n_x32 : P.g.n_xblk32, P.g.tpc32, st);
  return B2_ERR_ARG;
}
