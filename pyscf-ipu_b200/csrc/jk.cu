// J/K from the s8 unique-ERI list (sm_100a).
//
// Semantics of the reference's sparse symmetric einsum (sparse_symmetric_ERI.py:86-137,
// index table compute_indices.cpp:22-101): every unique (ij|kl) value is divided by its
// repetition count 2^(d_ij + d_kl + d_(ij,kl)) (num_repetitions_fast, lines 68-79) and
// applied through all 8 index permutations to J[k,l] = sum (ij|kl) D[j,i] and
// K[i,l] = sum (ij|kl) D[j,k] (nanoDFT.py:129-132).  With D symmetric the 8 permutations
// reduce to 2 J and 4 K updates of one accumulator followed by J = Jacc + Jacc^T,
// K = Kacc + Kacc^T.
//
// Decomposition: one CTA per chunk of one molecule's s8 list; D and the Jacc/Kacc
// accumulators live in shared memory (nao <= 70).  Each thread walks runs of 8 consecutive
// list entries (two 16-byte vector loads for float32 storage), decoding (i,j,k,l) once per
// run and then incrementally.  Partial sums whose target is fixed along the run stay in
// registers -- Jacc[i,j] for the row, Kacc[i,k] and Kacc[j,k] for a k-run -- and are added
// when the run leaves that row / k-run; Jacc[k,l], Kacc[i,l], Kacc[j,l] are added per entry.
// Every product and sum is float64 (ERIs may be stored in float32): the SCF map stays a
// smooth function of D, which keeps DIIS converging below the float32 rounding level.
//
// Accumulators.  64-bit shared-memory atomics (float64 or int64) are not native on sm_100a
// and dominate the kernel; 32-bit integer shared atomics are.  The float32-storage kernel
// therefore accumulates in fixed point: each addend x becomes q = rint(x * 2^36) (int64),
// split into three 32-bit words lo = q & 0x3fff, mid = (q >> 14) & 0x3fff, hi = q >> 28
// (arithmetic shift), each summed with a native 32-bit atomicAdd.  The sums are exact:
// one CTA makes at most 6 adds per list entry to one target, so the lo/mid sums stay
// below 6 * chunk * 2^14 < 2^32, and hi is exact modulo 2^32 while |partial| < 2^23
// (|ERI| < 8 and |D| < 4 bound it by 6 * chunk * 32 < 2^23 for chunk <= 32768).  The
// rounding (2^-37 per addend) is far below the float32 storage error of the ERIs and, being
// deterministic per addend, keeps the map smooth.  The float64-storage kernel keeps float64
// shared atomics, so the all-float64 path matches the reference to rounding.
#include "device_plan.cuh"

#define B2_JK_RUN 8

__device__ __forceinline__ long long b2_untri_fast(long long p) {
  long long i = (long long)((sqrtf(8.0f * (float)p + 1.0f) - 1.0f) * 0.5f);
  while ((i + 1) * (i + 2) / 2 <= p) ++i;
  while (i * (i + 1) / 2 > p) --i;
  return i;
}

template <typename T> struct B2Vec;
template <> struct B2Vec<float> {
  __device__ static void load8(const float *p, double *v) {
    const float4 a = *reinterpret_cast<const float4 *>(p);
    const float4 b = *reinterpret_cast<const float4 *>(p + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  }
};
template <> struct B2Vec<double> {
  __device__ static void load8(const double *p, double *v) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 a = *reinterpret_cast<const double2 *>(p + 2 * q);
      v[2 * q] = a.x; v[2 * q + 1] = a.y;
    }
  }
};

// Accumulator policies: float64 shared atomics, or the exact 3-word fixed point.
struct B2AccF64 {
  static constexpr int WORDS = 2;              // 32-bit words per element
  __device__ static void zero(unsigned *b, int nn, int e) { reinterpret_cast<double *>(b)[e] = 0.0; }
  __device__ static void add(unsigned *b, int nn, int e, double v) {
    atomicAdd(reinterpret_cast<double *>(b) + e, v);
  }
  __device__ static double get(const unsigned *b, int nn, int e) { return reinterpret_cast<const double *>(b)[e]; }
};
#define B2_JK_FX_SCALE 68719476736.0           // 2^36
struct B2AccFix3 {
  static constexpr int WORDS = 3;
  __device__ static void zero(unsigned *b, int nn, int e) { b[e] = 0u; b[nn + e] = 0u; b[2 * nn + e] = 0u; }
  __device__ static void add(unsigned *b, int nn, int e, double v) {
    const long long q = __double2ll_rn(v * B2_JK_FX_SCALE);
    atomicAdd(b + e, (unsigned)(q & 0x3FFF));
    atomicAdd(b + nn + e, (unsigned)((q >> 14) & 0x3FFF));
    atomicAdd(b + 2 * nn + e, (unsigned)(int)(q >> 28));
  }
  __device__ static double get(const unsigned *b, int nn, int e) {
    const long long q = ((long long)(int)b[2 * nn + e] << 28) + ((long long)b[nn + e] << 14) + (long long)b[e];
    return (double)q * (1.0 / B2_JK_FX_SCALE);
  }
};

template <typename T, typename A, int NT>
__global__ void __launch_bounds__(NT)
k_jk_s8(const B2MolDev *__restrict__ mols, const long long *__restrict__ chunk_off, int nmol,
        long long chunk, const int *__restrict__ active, const T *__restrict__ eri,
        const double *__restrict__ D, double *__restrict__ J, double *__restrict__ K,
        const int *__restrict__ mol_map) {
  extern __shared__ double smem_d[];
  const long long cid = blockIdx.x;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (chunk_off[mid] <= cid) lo = mid; else hi = mid - 1;
  }
  const int mol = mol_map ? mol_map[lo] : lo;
  if (active && !active[mol]) return;
  const B2MolDev md = mols[mol];
  const int N = md.nao, NN = N * N;
  double *sD = smem_d;
  unsigned *sJ = reinterpret_cast<unsigned *>(sD + NN), *sK = sJ + A::WORDS * NN;
  for (int e = threadIdx.x; e < NN; e += NT) {
    sD[e] = D[md.mat_off + e];
    A::zero(sJ, NN, e);
    A::zero(sK, NN, e);
  }
  __syncthreads();
  const long long p0 = (cid - chunk_off[lo]) * chunk;
  const long long p1 = min(p0 + chunk, md.n4);
  const T *E = eri + md.eri_off;
  for (long long base = p0 + (long long)threadIdx.x * B2_JK_RUN; base < p1;
       base += (long long)NT * B2_JK_RUN) {
    double v[B2_JK_RUN];
    B2Vec<T>::load8(E + base, v);
    // decode the first entry of the run
    long long ij = b2_untri_fast(base);
    int kl = (int)(base - ij * (ij + 1) / 2);
    int i = (int)b2_untri_fast(ij), j = (int)(ij - (long long)i * (i + 1) / 2);
    int k = (int)b2_untri_fast(kl), l = kl - k * (k + 1) / 2;
    double Dij = sD[i * N + j];
    double aJ = 0, aKi = 0, aKj = 0;
    const int nrun = (int)min((long long)B2_JK_RUN, p1 - base);
#pragma unroll
    for (int r = 0; r < B2_JK_RUN; ++r) {
      if (r < nrun) {
        double f = v[r];
        if (f != 0.0) {
          if (i == j) f *= 0.5;
          if (k == l) f *= 0.5;
          if (ij == kl) f *= 0.5;
          aJ += f * sD[k * N + l];
          aKi += f * sD[j * N + l];
          aKj += f * sD[i * N + l];
          A::add(sJ, NN, k * N + l, 2.0 * f * Dij);
          A::add(sK, NN, i * N + l, f * sD[j * N + k]);
          A::add(sK, NN, j * N + l, f * sD[i * N + k]);
        }
        const bool row_end = (kl == ij);
        const bool run_end = row_end || (l == k) || (r == nrun - 1);
        if (run_end) {                              // leave the k-run: flush its partials
          if (aKi != 0.0) A::add(sK, NN, i * N + k, aKi);
          if (aKj != 0.0) A::add(sK, NN, j * N + k, aKj);
          aKi = 0; aKj = 0;
        }
        if (row_end || r == nrun - 1) {             // leave the row: flush Jacc[i,j]
          if (aJ != 0.0) A::add(sJ, NN, i * N + j, 2.0 * aJ);
          aJ = 0;
        }
        if (row_end) {
          ++ij; kl = 0; k = 0; l = 0;
          if (++j > i) { ++i; j = 0; }
          Dij = sD[i * N + j < NN ? i * N + j : 0];
        } else {
          ++kl;
          if (l == k) { ++k; l = 0; } else { ++l; }
        }
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NN; e += NT) {
    const int a = e / N, b = e - (e / N) * N;
    const double jv = A::get(sJ, NN, a * N + b) + A::get(sJ, NN, b * N + a);
    const double kv = A::get(sK, NN, a * N + b) + A::get(sK, NN, b * N + a);
    if (jv != 0.0) atomicAdd(&J[md.mat_off + e], jv);
    if (kv != 0.0) atomicAdd(&K[md.mat_off + e], kv);
  }
}

__global__ void k_zero_active(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
                              double *__restrict__ A, double *__restrict__ B) {
  const int m = blockIdx.x;
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  for (int e = threadIdx.x; e < md.nao * md.nao; e += blockDim.x) {
    A[md.mat_off + e] = 0.0;
    if (B) B[md.mat_off + e] = 0.0;
  }
}

int b2_zero_active(const B2PlanDev &P, const int *active, double *A, double *B, cudaStream_t st) {
  k_zero_active<<<P.h.nmol, 256, 0, st>>>(P.mols, active, A, B);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_jk_s8(const B2PlanDev &P, int precision, const int *active, const void *eri,
                    const double *D, double *J, double *K, cudaStream_t st) {
  if (P.jk_nchunks <= 0) return B2_OK;
  const bool sub = P.sub.n > 0;
  const long long *coff = sub ? P.sub.jk_off : P.jk_chunk_off;
  const int nm = sub ? P.sub.n : P.h.nmol;
  const long long nch = sub ? P.sub.jk_n : P.jk_nchunks;
  const int *map = sub ? P.sub.mol_map : nullptr;
  if (nch <= 0) return B2_OK;
  if (active) {
    int rc = b2_zero_active(P, active, J, K, st);
    if (rc) return rc;
  } else {
    B2_CUDA_TRY(cudaMemsetAsync(J, 0, sizeof(double) * P.h.n_mat, st));
    B2_CUDA_TRY(cudaMemsetAsync(K, 0, sizeof(double) * P.h.n_mat, st));
  }
  const int N = P.h.max_nao;
  if (precision == 64) {
    constexpr int NT = 512;
    if (P.jk_chunk % (NT * B2_JK_RUN) != 0) return B2_ERR_ARG;
    const size_t sm = sizeof(double) * N * N + 4u * (2 * B2AccF64::WORDS) * N * N;
    auto kern = k_jk_s8<double, B2AccF64, NT>;
    B2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<(unsigned)nch, NT, sm, st>>>(P.mols, coff, nm, P.jk_chunk, active, (const double *)eri, D, J, K, map);
  } else if (precision == 32) {
    constexpr int NT = 1024;
    if (P.jk_chunk % (NT * B2_JK_RUN) != 0 || P.jk_chunk > 32768) return B2_ERR_ARG;
    const size_t sm = sizeof(double) * N * N + 4u * (2 * B2AccFix3::WORDS) * N * N;
    auto kern = k_jk_s8<float, B2AccFix3, NT>;
    B2_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<(unsigned)nch, NT, sm, st>>>(P.mols, coff, nm, P.jk_chunk, active, (const float *)eri, D, J, K, map);
  } else {
    return B2_ERR_ARG;
  }
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
