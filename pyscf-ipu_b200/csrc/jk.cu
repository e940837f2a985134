// J/K from the s8 unique-ERI list (sm_100a).
//
// Semantics of the reference's sparse symmetric einsum (sparse_symmetric_ERI.py:86-137,
// index table compute_indices.cpp:22-101): every unique (ij|kl) value is divided by its
// repetition count 2^(d_ij + d_kl + d_(ij,kl)) (num_repetitions_fast, lines 68-79) and
// applied through all 8 index permutations to J[k,l] = sum (ij|kl) D[j,i] and
// K[i,l] = sum (ij|kl) D[j,k] (nanoDFT.py:129-132).  With D symmetric the 8 permutations
// reduce to 2 J and 4 K updates of one triangle-agnostic accumulator followed by
// J = Jacc + Jacc^T, K = Kacc + Kacc^T.
//
// Decomposition: one CTA per chunk of one molecule's s8 list.  D, Jacc and Kacc live in
// shared memory (nao <= 70), ERIs stream from HBM once with coalesced loads; the index
// quadruple is decoded from the list position in registers (no index arrays, unlike the
// reference's int16 index tensors, nanoDFT.py:310-313).  Each CTA adds its partial J and K
// to global memory at the end.
#include "device_plan.cuh"

__device__ __forceinline__ long long b2_untri_fast(long long p) {
  long long i = (long long)((sqrtf(8.0f * (float)p + 1.0f) - 1.0f) * 0.5f);
  while ((i + 1) * (i + 2) / 2 <= p) ++i;
  while (i * (i + 1) / 2 > p) --i;
  return i;
}

template <typename T>
__global__ void __launch_bounds__(256)
k_jk_s8(const B2MolDev *__restrict__ mols, const long long *__restrict__ chunk_off, int nmol,
        long long chunk, const T *__restrict__ eri, const double *__restrict__ D,
        double *__restrict__ J, double *__restrict__ K) {
  extern __shared__ unsigned char smem_raw[];
  T *sD = reinterpret_cast<T *>(smem_raw);
  const long long cid = blockIdx.x;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (chunk_off[mid] <= cid) lo = mid; else hi = mid - 1;
  }
  const B2MolDev md = mols[lo];
  const int N = md.nao, NN = N * N;
  T *sJ = sD + NN;
  T *sK = sJ + NN;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    sD[e] = (T)D[md.mat_off + e];
    sJ[e] = (T)0;
    sK[e] = (T)0;
  }
  __syncthreads();
  const long long p0 = (cid - chunk_off[lo]) * chunk;
  const long long p1 = min(p0 + chunk, md.n4);
  const T *E = eri + md.eri_off;
  for (long long p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    T v = E[p];
    if (v == (T)0) continue;
    const long long ij = b2_untri_fast(p);
    const int kl = (int)(p - ij * (ij + 1) / 2);
    const int i = (int)b2_untri_fast(ij);
    const int j = (int)(ij - (long long)i * (i + 1) / 2);
    const int k = (int)b2_untri_fast(kl);
    const int l = kl - k * (k + 1) / 2;
    if (i == j) v *= (T)0.5;
    if (k == l) v *= (T)0.5;
    if (ij == kl) v *= (T)0.5;
    const T v2 = v + v;
    atomicAdd(&sJ[i * N + j], v2 * sD[k * N + l]);
    atomicAdd(&sJ[k * N + l], v2 * sD[i * N + j]);
    atomicAdd(&sK[i * N + k], v * sD[j * N + l]);
    atomicAdd(&sK[i * N + l], v * sD[j * N + k]);
    atomicAdd(&sK[j * N + k], v * sD[i * N + l]);
    atomicAdd(&sK[j * N + l], v * sD[i * N + k]);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    const T jv = sJ[a * N + b] + sJ[b * N + a];
    const T kv = sK[a * N + b] + sK[b * N + a];
    if (jv != (T)0) atomicAdd(&J[md.mat_off + e], (double)jv);
    if (kv != (T)0) atomicAdd(&K[md.mat_off + e], (double)kv);
  }
}

int b2_launch_jk_s8(const B2PlanDev &P, int precision, const void *eri, const double *D, double *J,
                    double *K, cudaStream_t st) {
  if (P.jk_nchunks <= 0) return B2_OK;
  B2_CUDA_TRY(cudaMemsetAsync(J, 0, sizeof(double) * P.h.n_mat, st));
  B2_CUDA_TRY(cudaMemsetAsync(K, 0, sizeof(double) * P.h.n_mat, st));
  const int N = P.h.max_nao;
  if (precision == 64) {
    size_t sm = sizeof(double) * 3 * N * N;
    B2_CUDA_TRY(cudaFuncSetAttribute(k_jk_s8<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_jk_s8<double><<<(unsigned)P.jk_nchunks, 256, sm, st>>>(P.mols, P.jk_chunk_off, P.h.nmol,
                                                            P.jk_chunk, (const double *)eri, D, J, K);
  } else if (precision == 32) {
    size_t sm = sizeof(float) * 3 * N * N;
    B2_CUDA_TRY(cudaFuncSetAttribute(k_jk_s8<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_jk_s8<float><<<(unsigned)P.jk_nchunks, 256, sm, st>>>(P.mols, P.jk_chunk_off, P.h.nmol,
                                                           P.jk_chunk, (const float *)eri, D, J, K);
  } else {
    return B2_ERR_ARG;
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
