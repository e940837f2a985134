// J/K as two symmetric matrix-vector products over s8-packed arrays (sm_100a).
//
// Same J and K as k_jk_s8 (J[k,l] = sum_ij (ij|kl) D[i,j], K[i,l] = sum_jk (ij|kl) D[j,k],
// nanoDFT.py:129-132; s8 semantics sparse_symmetric_ERI.py:86-137), restated so that every
// list entry feeds registers instead of scattered shared-memory atomics:
//
//   J_pair = M x_J,  M[(ij),(kl)] = (ij|kl)                 (the s8 list itself)
//   K_pair = H x_K,  H[(il),(jk)] = (ij|kl) + (ik|jl)        (the exchange list)
//   x_J[(ij)] = D[i,j] (2 - d_ij),   x_K[(jk)] = D[j,k] (1 - d_jk / 2)
//
// with pairs (ij), i >= j, indexed ij = i(i+1)/2 + j.  Both M and H are symmetric in their two
// pair indices (H[(jk),(il)] = (ji|lk) + (jl|ik) = H[(il),(jk)]), so H is stored exactly like the
// s8 list: row P = (il), columns Q <= P, packed row after row.  K follows from splitting the
// sum over ordered (j,k) into j > k, j < k (relabelled) and j = k.
//
// The exchange list is built once per ERI list (k_exch_build: two gathers per entry from the
// molecule's s8 list, which stays in L2).  The product kernel (k_symv) gives each warp a strip
// of 128 columns and a block of 64 rows of one molecule: lanes own 4 columns each and copy every
// row segment with coalesced cp.async into a 3-stage shared-memory ring (groups of 8 rows, two
// groups in flight while one is reduced), keep the column sums y[Q] += A[P,Q] x[P] in float64
// registers for the whole block and reduce the row sums y[P] += sum_Q A[P,Q] x[Q] of 8 rows at
// a time with one transposed butterfly of warp shuffles; one float64 global atomic per row per
// strip and per column per block.  Every product and sum is float64 (the lists may be stored in
// float32).  Algorithmic bytes per call: 2 n4 sizeof(T) per molecule (both lists once).
#include "device_plan.cuh"

#define B2_SV_STRIP 128
#define B2_SV_ROWS 64
#define B2_SV_GROUP 8           // rows per copy group (the row-sum butterfly is written for 8)
#define B2_SV_STAGES 3          // copy groups in each warp's shared-memory ring
#define B2_SV_WARPS 4           // warps (tasks) per CTA

__device__ __forceinline__ long long b2_sv_untri(long long p) {
  long long i = (long long)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= p) ++i;
  while (i * (i + 1) / 2 > p) --i;
  return i;
}
__device__ __forceinline__ long long b2_sv_idx(int a, int b, int c, int d) {   // s8 index of (ab|cd)
  const long long p = a >= b ? b2_tri(a) + b : b2_tri(b) + a;
  const long long q = c >= d ? b2_tri(c) + d : b2_tri(d) + c;
  return p >= q ? b2_tri(p) + q : b2_tri(q) + p;
}

// exchange list from the s8 list; CTA = one J/K chunk (same chunks as k_jk_s8)
template <typename T>
__global__ void __launch_bounds__(256)
k_exch_build(const B2MolDev *__restrict__ mols, const long long *__restrict__ chunk_off, int nmol,
             long long chunk, const T *__restrict__ eri, T *__restrict__ exch) {
  const long long cid = blockIdx.x;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (chunk_off[mid] <= cid) lo = mid; else hi = mid - 1;
  }
  const B2MolDev md = mols[lo];
  const long long p0 = (cid - chunk_off[lo]) * chunk, p1 = min(p0 + chunk, md.n4);
  const T *E = eri + md.eri_off;
  T *X = exch + md.eri_off;
  // runs of 8 consecutive entries per thread: decode (i,l | j,k) once, then step
  for (long long e0 = p0 + 8 * (long long)threadIdx.x; e0 < p1; e0 += 8 * (long long)blockDim.x) {
    long long P = b2_sv_untri(e0), Q = e0 - b2_tri(P);
    int i = (int)b2_sv_untri(P), l = (int)(P - b2_tri(i));
    int j = (int)b2_sv_untri(Q), k = (int)(Q - b2_tri(j));
    const int n = (int)min(8ll, p1 - e0);
    for (int r = 0; r < n; ++r) {
      X[e0 + r] = E[b2_sv_idx(i, j, k, l)] + E[b2_sv_idx(i, k, j, l)];
      if (Q == P) {                 // next row (il): Q = 0, (j,k) = (0,0)
        ++P; Q = 0; j = 0; k = 0;
        if (++l > i) { ++i; l = 0; }
      } else {
        ++Q;
        if (++k > j) { ++j; k = 0; }
      }
    }
  }
}

// per active molecule: x_J, x_K (pair-indexed) from D, y_J = y_K = 0
__global__ void k_sv_x(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
                       const int *__restrict__ mol_map, const double *__restrict__ D,
                       double *__restrict__ xJ, double *__restrict__ xK, double *__restrict__ yJ,
                       double *__restrict__ yK) {
  const int m = mol_map ? mol_map[blockIdx.x] : blockIdx.x;
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  const int N = md.nao;
  const int n2 = N * (N + 1) / 2;
  for (int P = threadIdx.x; P < n2; P += blockDim.x) {
    const int i = (int)b2_sv_untri(P), j = P - (int)b2_tri(i);
    const double d = D[md.mat_off + (long long)i * N + j];
    xJ[md.row_off + P] = i == j ? d : 2.0 * d;
    xK[md.row_off + P] = i == j ? 0.5 * d : d;
    yJ[md.row_off + P] = 0.0;
    yK[md.row_off + P] = 0.0;
  }
}

// warp tasks of one molecule: strips of 128 columns, each cut into blocks of 64 rows (P >= Q)
__host__ __device__ inline long long b2_sv_tasks(long long n2) {
  long long t = 0;
  for (long long q0 = 0; q0 < n2; q0 += B2_SV_STRIP) t += (n2 - q0 + B2_SV_ROWS - 1) / B2_SV_ROWS;
  return t;
}

// cp.async of one list entry into shared memory (zero fill when !ok; the address is then
// not read but kept valid)
template <int B>
__device__ __forceinline__ void b2_cp_async(uint32_t dst, const void *src, bool ok);
template <>
__device__ __forceinline__ void b2_cp_async<4>(uint32_t dst, const void *src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"(dst), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
template <>
__device__ __forceinline__ void b2_cp_async<8>(uint32_t dst, const void *src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" :: "r"(dst), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void b2_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void b2_cp_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }

// copies of one row group (rows P0.. of the row block ending at r1, zero beyond it) into a
// stage [B2_SV_GROUP][B2_SV_STRIP] of the warp's ring; each lane copies exactly the entries
// it reads later (its 4 columns), so no cross-lane synchronisation is needed.  Pair indices
// are int: a molecule's pair count n2 <= 3240 keeps tri(P) < 2^23.
template <typename T>
__device__ __forceinline__ void b2_sv_issue(const T *__restrict__ A, int P0, int r1, const int (&qc)[4],
                                            uint32_t stage, int lane) {
#pragma unroll
  for (int rr = 0; rr < B2_SV_GROUP; ++rr) {
    const int P = P0 + rr;
    const T *row = A + (P * (P + 1) >> 1);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const bool ok = P < r1 && qc[c] <= P;
      b2_cp_async<sizeof(T)>(stage + (uint32_t)((rr * B2_SV_STRIP + lane + 32 * c) * sizeof(T)),
                             ok ? (const void *)(row + qc[c]) : (const void *)A, ok);
    }
  }
}

// one row group: column sums into yc, row sums reduced over the warp and added to y
template <typename T>
__device__ __forceinline__ void b2_sv_use(const T *__restrict__ st, const double *__restrict__ x, int P0,
                                          int r1, const int (&qc)[4], const double (&xq)[4], double (&yc)[4],
                                          double *__restrict__ y, int lane) {
  double rs[B2_SV_GROUP];
#pragma unroll
  for (int rr = 0; rr < B2_SV_GROUP; ++rr) {
    const int P = P0 + rr;
    const double xp = P < r1 ? x[P] : 0.0;
    rs[rr] = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double av = (double)st[rr * B2_SV_STRIP + lane + 32 * c];
      rs[rr] += av * xq[c];
      if (qc[c] < P) yc[c] += av * xp;
    }
  }
  // transposed butterfly: each step hands half of the remaining rows to the partner lane,
  // 4 + 2 + 1 + 1 + 1 shuffles for the 8 rows; lane 4r ends with the warp total of row r
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
  double s4[4], s2[2];
#pragma unroll
  for (int k = 0; k < 4; ++k)                  // s4[k]: row (h16 ? 4 : 0) + k
    s4[k] = (h16 ? rs[k + 4] : rs[k]) + __shfl_xor_sync(0xffffffffu, h16 ? rs[k] : rs[k + 4], 16);
#pragma unroll
  for (int k = 0; k < 2; ++k)                  // s2[k]: row (h16 ? 4 : 0) + (h8 ? 2 : 0) + k
    s2[k] = (h8 ? s4[k + 2] : s4[k]) + __shfl_xor_sync(0xffffffffu, h8 ? s4[k] : s4[k + 2], 8);
  double s1 = (h4 ? s2[1] : s2[0]) + __shfl_xor_sync(0xffffffffu, h4 ? s2[0] : s2[1], 4);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
  s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
  if ((lane & 3) == 0 && P0 + (lane >> 2) < r1 && s1 != 0.0) atomicAdd(&y[P0 + (lane >> 2)], s1);
}

template <typename T>
__host__ __device__ constexpr int b2_sv_smem() {    // bytes per CTA
  return B2_SV_WARPS * B2_SV_STAGES * B2_SV_GROUP * B2_SV_STRIP * (int)sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(32 * B2_SV_WARPS)
k_symv(const B2MolDev *__restrict__ mols, const long long *__restrict__ task_off, int nmol,
       const int *__restrict__ active, const int *__restrict__ mol_map, const T *__restrict__ eri,
       const T *__restrict__ exch, const double *__restrict__ xJ, const double *__restrict__ xK,
       double *__restrict__ yJ, double *__restrict__ yK) {
  extern __shared__ __align__(16) unsigned char sv_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long t = (long long)blockIdx.x * B2_SV_WARPS + w;
  if (t >= task_off[nmol]) return;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (task_off[mid] <= t) lo = mid; else hi = mid - 1;
  }
  const int m = mol_map ? mol_map[lo] : lo;
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  const int n2 = md.nao * (md.nao + 1) / 2;
  // blockIdx.y: 0 = J (s8 list, x_J), 1 = K (exchange list, x_K)
  const T *A = (blockIdx.y == 0 ? eri : exch) + md.eri_off;
  const double *x = (blockIdx.y == 0 ? xJ : xK) + md.row_off;
  double *y = (blockIdx.y == 0 ? yJ : yK) + md.row_off;
  int u = (int)(t - task_off[lo]), q0 = 0;
  for (;;) {                                   // strip and row block of local task u
    const int nb = (n2 - q0 + B2_SV_ROWS - 1) / B2_SV_ROWS;
    if (u < nb) break;
    u -= nb;
    q0 += B2_SV_STRIP;
  }
  const int r0 = q0 + u * B2_SV_ROWS, r1 = min(r0 + B2_SV_ROWS, n2);
  int qc[4];
  double xq[4], yc[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    qc[c] = q0 + lane + 32 * c;
    xq[c] = qc[c] < n2 ? x[qc[c]] : 0.0;
    yc[c] = 0.0;
  }
  // ring of B2_SV_STAGES row groups per warp: group g + STAGES - 1 is copied while group g is
  // reduced (the kernel is bound by memory latency otherwise)
  constexpr int SB = B2_SV_GROUP * B2_SV_STRIP;                   // entries per stage
  T *ring = reinterpret_cast<T *>(sv_smem) + (size_t)w * B2_SV_STAGES * SB;
  const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring);
  const int ng = (r1 - r0 + B2_SV_GROUP - 1) / B2_SV_GROUP;
#pragma unroll
  for (int g = 0; g < B2_SV_STAGES - 1; ++g) {
    if (g < ng) b2_sv_issue(A, r0 + g * B2_SV_GROUP, r1, qc, ring_s + (uint32_t)(g * SB * sizeof(T)), lane);
    b2_cp_commit();
  }
  for (int g = 0; g < ng; ++g) {
    const int gn = g + B2_SV_STAGES - 1;
    if (gn < ng)
      b2_sv_issue(A, r0 + gn * B2_SV_GROUP, r1, qc, ring_s + (uint32_t)((gn % B2_SV_STAGES) * SB * sizeof(T)), lane);
    b2_cp_commit();
    b2_cp_wait<B2_SV_STAGES - 1>();            // this lane's copies of group g have landed
    b2_sv_use(ring + (g % B2_SV_STAGES) * SB, x, r0 + g * B2_SV_GROUP, r1, qc, xq, yc, y, lane);
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (qc[c] < n2 && yc[c] != 0.0) atomicAdd(&y[qc[c]], yc[c]);
}

// J, K (nao x nao) of the active molecules from the pair-indexed results
__global__ void k_sv_out(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
                         const int *__restrict__ mol_map, const double *__restrict__ yJ,
                         const double *__restrict__ yK, double *__restrict__ J, double *__restrict__ K) {
  const int m = mol_map ? mol_map[blockIdx.x] : blockIdx.x;
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  const int N = md.nao;
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    const long long P = a >= b ? b2_tri(a) + b : b2_tri(b) + a;
    J[md.mat_off + e] = yJ[md.row_off + P];
    K[md.mat_off + e] = yK[md.row_off + P];
  }
}

int b2_launch_exch_build(const B2PlanDev &P, int precision, const void *eri, void *exch, cudaStream_t st) {
  if (P.jk_nchunks <= 0) return B2_OK;
  if (precision == 64)
    k_exch_build<double><<<(unsigned)P.jk_nchunks, 256, 0, st>>>(P.mols, P.jk_chunk_off, P.h.nmol, P.jk_chunk,
                                                                 (const double *)eri, (double *)exch);
  else if (precision == 32)
    k_exch_build<float><<<(unsigned)P.jk_nchunks, 256, 0, st>>>(P.mols, P.jk_chunk_off, P.h.nmol, P.jk_chunk,
                                                                (const float *)eri, (float *)exch);
  else
    return B2_ERR_ARG;
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_jk_symv(const B2PlanDev &P, int precision, const int *active, const void *eri,
                      const void *exch, const double *D, double *J, double *K, double *work,
                      cudaStream_t st) {
  if (precision != 64 && precision != 32) return B2_ERR_ARG;
  const bool sub = P.sub.n > 0;
  const int nm = sub ? P.sub.n : P.h.nmol;
  const int *map = sub ? P.sub.mol_map : nullptr;
  const long long *toff = sub ? P.sub.sv_off : P.sv_off;
  const long long ntask = sub ? P.sub.sv_n : P.sv_ntask;
  if (nm <= 0) return B2_OK;
  const long long nr = P.h.n_rows;
  double *xJ = work, *xK = xJ + nr, *yJ = xK + nr, *yK = yJ + nr;
  k_sv_x<<<nm, 256, 0, st>>>(P.mols, active, map, D, xJ, xK, yJ, yK);
  b2_count_launches(1);
  if (ntask > 0) {
    const dim3 grid((unsigned)((ntask + B2_SV_WARPS - 1) / B2_SV_WARPS), 2);
    if (precision == 64) {
      B2_CUDA_TRY(cudaFuncSetAttribute(k_symv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       b2_sv_smem<double>()));
      k_symv<double><<<grid, 32 * B2_SV_WARPS, b2_sv_smem<double>(), st>>>(
          P.mols, toff, nm, active, map, (const double *)eri, (const double *)exch, xJ, xK, yJ, yK);
    } else {
      B2_CUDA_TRY(cudaFuncSetAttribute(k_symv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       b2_sv_smem<float>()));
      k_symv<float><<<grid, 32 * B2_SV_WARPS, b2_sv_smem<float>(), st>>>(
          P.mols, toff, nm, active, map, (const float *)eri, (const float *)exch, xJ, xK, yJ, yK);
    }
    b2_count_launches(1);
  }
  k_sv_out<<<nm, 256, 0, st>>>(P.mols, active, map, yJ, yK, J, K);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

long long b2_sv_tasks_host(long long n2) { return b2_sv_tasks(n2); }
