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
// of 128 columns and a block of 128 rows of one molecule: lanes own 4 columns each; every row
// segment arrives by one bulk copy (8 lanes issue a group's 8 rows) in a 2-stage shared-memory
// ring (groups of 8 rows: the next group is in flight while one is reduced; 3 CTAs of 8 warps
// per SM), keep the column sums y[Q] += A[P,Q] x[P] in float64
// registers for the whole block and reduce the row sums y[P] += sum_Q A[P,Q] x[Q] of 8 rows at
// a time with one transposed butterfly of warp shuffles; one float64 global atomic per row per
// strip and per column per block.  Every product and sum is float64 (the lists may be stored in
// float32).  Algorithmic bytes per call: 2 n4 sizeof(T) per molecule (both lists once).
#include "device_plan.cuh"

#define B2_SV_STRIP 128
#ifndef B2_SV_ROWS
#define B2_SV_ROWS 128          // rows per warp task
#endif
#define B2_SV_GROUP 8           // rows per copy group (the row-sum butterfly is written for 8)
#ifndef B2_SV_STAGES
#define B2_SV_STAGES 2          // copy groups in each warp's shared-memory ring
#endif
#ifndef B2_SV_WARPS
#define B2_SV_WARPS 8           // warps (tasks) per CTA
#endif

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
    // all 16 gather addresses first, then the loads (8 entries' gathers in flight together)
    long long ia[8], ib[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      ia[r] = b2_sv_idx(i, j, k, l);
      ib[r] = b2_sv_idx(i, k, j, l);
      if (Q == P) {                 // next row (il): Q = 0, (j,k) = (0,0)
        ++P; Q = 0; j = 0; k = 0;
        if (++l > i) { ++i; l = 0; }
      } else {
        ++Q;
        if (++k > j) { ++j; k = 0; }
      }
    }
    T va[8], vb[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      va[r] = r < n ? E[ia[r]] : (T)0;
      vb[r] = r < n ? E[ib[r]] : (T)0;
    }
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (r < n) X[e0 + r] = va[r] + vb[r];
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

// warp tasks of one molecule: strips of 128 columns, each cut into blocks of B2_SV_ROWS rows (P >= Q)
__host__ __device__ inline long long b2_sv_tasks(long long n2) {
  long long t = 0;
  for (long long q0 = 0; q0 < n2; q0 += B2_SV_STRIP) t += (n2 - q0 + B2_SV_ROWS - 1) / B2_SV_ROWS;
  return t;
}

__device__ int g_b2_sv_err = 0;   // 1: a wait on a row-group copy gave up (status: b2_jk_status)

#define B2_SV_SPIN (1 << 22)       // polls of an mbarrier before a wait gives up

__device__ __forceinline__ void b2_sv_mbar_init(uint32_t a) {     // one arrival per row of a group
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(a), "n"(B2_SV_GROUP) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void b2_sv_expect(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void b2_sv_bulk(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}
__device__ __forceinline__ bool b2_sv_wait(uint32_t a, uint32_t parity) {
  for (int it = 0; it < B2_SV_SPIN; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}

// Row segments of one row group (rows P0.., the row block ends at r1) -> one stage of the warp's
// ring: lane rr < B2_SV_GROUP copies row P0 + rr with one bulk copy of A[P, q0 .. min(q0+128,
// P+1)), widened to the 16-byte-aligned bytes around it (the molecule's list starts 128-byte
// aligned and is padded to a multiple of 32 entries, so the widened range stays inside it), and
// arrives on the stage's mbarrier (8 arrivals, each expecting its own bytes; a lane without a row
// arrives expecting none).  Row rr lands at byte rr * b2_sv_rb of the stage with its first entry
// at in-row offset (tri(P) + q0) mod (16 / sizeof(T)).  Pair indices are int: n2 <= 3240 keeps
// tri(P) < 2^23.
template <typename T>
__host__ __device__ constexpr int b2_sv_rb() { return B2_SV_STRIP * (int)sizeof(T) + 32; }   // row bytes
template <typename T>
__device__ __forceinline__ void b2_sv_issue(const T *__restrict__ A, int P0, int r1, int q0, uint32_t stage,
                                            uint32_t mbar, int lane) {
  if (lane >= B2_SV_GROUP) return;
  const int P = P0 + lane;
  uint32_t bytes = 0;
  long long a0 = 0;
  if (P < r1) {
    const long long e0 = (P * (P + 1) >> 1) + q0;
    const long long b0 = e0 * (long long)sizeof(T);
    const long long b1 = (e0 + min(q0 + B2_SV_STRIP, P + 1) - q0) * (long long)sizeof(T);
    a0 = b0 & ~15ll;
    bytes = (uint32_t)(((b1 + 15) & ~15ll) - a0);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  b2_sv_expect(mbar, bytes);
  if (bytes) b2_sv_bulk(stage + (uint32_t)(lane * b2_sv_rb<T>()), reinterpret_cast<const char *>(A) + a0, bytes, mbar);
}

// one row group from its stage: column sums into yc, row sums reduced over the warp into y.
// FULL: every row of the group is in the block and lies below the strip (P >= q0 + 128), so all
// 128 columns are present and off-diagonal: no masks.
template <typename T, bool FULL>
__device__ __forceinline__ void b2_sv_use(const unsigned char *__restrict__ stage, const double *__restrict__ x,
                                          int P0, int r1, int q0, const int (&qc)[4], const double (&xq)[4],
                                          double (&yc)[4], double *__restrict__ y, int lane) {
  constexpr int MSK = 16 / (int)sizeof(T) - 1;
  double rs[B2_SV_GROUP];
  int off = ((P0 * (P0 + 1) >> 1) + q0) & MSK;  // in-row offset of the row's first entry
#pragma unroll
  for (int rr = 0; rr < B2_SV_GROUP; ++rr) {
    const int P = P0 + rr;
    const T *row = reinterpret_cast<const T *>(stage + rr * b2_sv_rb<T>()) + off;
    off = (off + P + 1) & MSK;                   // tri(P + 1) = tri(P) + P + 1
    rs[rr] = 0.0;
    if (FULL) {
      const double xp = x[P];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const double av = (double)row[lane + 32 * c];
        rs[rr] += av * xq[c];
        yc[c] += av * xp;
      }
    } else {
      const bool ok = P < r1;
      const double xp = ok ? x[P] : 0.0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        // entries past the row's end (Q > P) and rows past the block are not copied: masked
        const double av = (ok && qc[c] <= P) ? (double)row[lane + 32 * c] : 0.0;
        rs[rr] += av * xq[c];
        if (qc[c] < P) yc[c] += av * xp;
      }
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
__host__ __device__ constexpr int b2_sv_stage_bytes() { return B2_SV_GROUP * b2_sv_rb<T>(); }
template <typename T>
__host__ __device__ constexpr int b2_sv_smem() {    // bytes per CTA: the rings, then the mbarriers
  return B2_SV_WARPS * B2_SV_STAGES * (b2_sv_stage_bytes<T>() + 8);
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
  constexpr int SB = b2_sv_stage_bytes<T>();
  unsigned char *ring = sv_smem + (size_t)w * B2_SV_STAGES * SB;
  const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring);
  const uint32_t mbar_s = (uint32_t)__cvta_generic_to_shared(sv_smem + B2_SV_WARPS * B2_SV_STAGES * SB) +
                          8u * (uint32_t)(w * B2_SV_STAGES);
  const int ng = (r1 - r0 + B2_SV_GROUP - 1) / B2_SV_GROUP;
  if (lane == 0)
    for (int k = 0; k < B2_SV_STAGES; ++k) b2_sv_mbar_init(mbar_s + 8u * k);
  __syncwarp();
  for (int g = 0; g < B2_SV_STAGES - 1 && g < ng; ++g)
    b2_sv_issue(A, r0 + g * B2_SV_GROUP, r1, q0, ring_s + (uint32_t)(g * SB), mbar_s + 8u * g, lane);
  int g = 0;
  for (; g < ng; ++g) {
    const int gn = g + B2_SV_STAGES - 1, sn = gn % B2_SV_STAGES, sc = g % B2_SV_STAGES;
    __syncwarp();                              // every lane is done with stage sn (group g - 1)
    if (gn < ng) b2_sv_issue(A, r0 + gn * B2_SV_GROUP, r1, q0, ring_s + (uint32_t)(sn * SB), mbar_s + 8u * sn, lane);
    const bool landed = b2_sv_wait(mbar_s + 8u * sc, (uint32_t)((g / B2_SV_STAGES) & 1));
    if (!__all_sync(0xffffffffu, landed)) {    // warp-uniform: the reduction below needs every lane
      if (lane == 0) atomicExch(&g_b2_sv_err, 1);
      break;
    }
    const int P0 = r0 + g * B2_SV_GROUP;
    if (r0 >= q0 + B2_SV_STRIP && P0 + B2_SV_GROUP <= r1)
      b2_sv_use<T, true>(ring + sc * SB, x, P0, r1, q0, qc, xq, yc, y, lane);
    else
      b2_sv_use<T, false>(ring + sc * SB, x, P0, r1, q0, qc, xq, yc, y, lane);
  }
  if (g < ng) {
    // gave up: wait (bounded) for the copies still in flight into this warp's ring, then leave
    for (int k = g; k < ng && k < g + B2_SV_STAGES; ++k)
      b2_sv_wait(mbar_s + 8u * (k % B2_SV_STAGES), (uint32_t)((k / B2_SV_STAGES) & 1));
    return;
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
  // the product kernel bulk-copies row segments widened to 16-byte boundaries: both lists must
  // start 16-byte aligned (every molecule's list then starts 128-byte aligned)
  if ((reinterpret_cast<uintptr_t>(eri) | reinterpret_cast<uintptr_t>(exch)) & 15) return B2_ERR_ARG;
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

int b2_jk_status_read(int reset) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_b2_sv_err, sizeof(int)) != cudaSuccess) return -1;
  if (reset) {
    const int z = 0;
    if (cudaMemcpyToSymbol(g_b2_sv_err, &z, sizeof(int)) != cudaSuccess) return -1;
  }
  return v;
}
