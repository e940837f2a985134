// Kernels of the learned initial-guess network (training and inference), sm_100a.
//
// The reference starts every SCF from the MINAO guess (pyscf_utils/minao.py:5-123); this
// project adds a message-passing network that predicts the initial density matrix per atom-pair
// block from the geometry (architecture and block parameterisation: oracle/nn_oracle.py, which
// is also the numpy check of these kernels).  Activations and master weights are float32;
// every matrix product rounds its inputs to bfloat16 (round to nearest even) and accumulates in
// float32 ("BF16 with FP32 accumulation").  All products go through one strided tiled GEMM.
#include <cuda_bf16.h>
#include "device_plan.cuh"

__device__ __forceinline__ float b2_bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// C[M x N] = beta * C + op(A) op(B) (+ bias[N]); A(i,k) = A[i*sai + k*sak], B(k,j) = B[k*sbk + j*sbj]
#define NN_BM 64
#define NN_BN 64
#define NN_BK 16
__global__ void __launch_bounds__(256)
k_nn_gemm(int M, int N, int K, const float *__restrict__ A, long long sai, long long sak,
          const float *__restrict__ B, long long sbk, long long sbj, float *__restrict__ C,
          long long ldc, const float *__restrict__ bias, float beta, int bf16) {
  __shared__ float As[NN_BK][NN_BM + 4];
  __shared__ float Bs[NN_BK][NN_BN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.y * NN_BM, j0 = blockIdx.x * NN_BN;
  float acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.f;
  for (int k0 = 0; k0 < K; k0 += NN_BK) {
    for (int e = threadIdx.x; e < NN_BK * NN_BM; e += 256) {
      const int kk = e / NN_BM, ii = e % NN_BM;
      const int gi = i0 + ii, gk = k0 + kk;
      float v = (gi < M && gk < K) ? A[gi * sai + gk * sak] : 0.f;
      As[kk][ii] = bf16 ? b2_bf16r(v) : v;
    }
    for (int e = threadIdx.x; e < NN_BK * NN_BN; e += 256) {
      const int kk = e / NN_BN, jj = e % NN_BN;
      const int gj = j0 + jj, gk = k0 + kk;
      float v = (gj < N && gk < K) ? B[gk * sbk + gj * sbj] : 0.f;
      Bs[kk][jj] = bf16 ? b2_bf16r(v) : v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < NN_BK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = As[kk][ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] += a[r] * b[c];
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int gi = i0 + ty + 16 * r, gj = j0 + tx + 16 * c;
      if (gi < M && gj < N) {
        float v = acc[r][c] + (bias ? bias[gj] : 0.f);
        float *dst = C + gi * ldc + gj;
        *dst = beta != 0.f ? beta * *dst + v : v;
      }
    }
}

// Tensor-core form of the same product (the one the network uses): bf16 inputs rounded to nearest even, fp32
// accumulation in tensor memory.  CTA tile 128 x 128, K step 64, two shared-memory stages: all
// 256 threads convert the next stage's float32 operands to bf16 while the tensor core works on
// the current one (one thread issues tcgen05.mma.kind::f16, M = 128, N = 128, K = 16, and commits
// to the stage's mbarrier).  Operands are K-major without swizzle: 8-row x 16-byte core matrices,
// element (row r, k) of a stage tile at byte ((k / 8) * 16 + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// (LBO 2048 B between k chunks, SBO 128 B between row groups).  Epilogue: warp w reads tensor
// memory lanes 32 (w % 4) .. + 31 (its rows) and columns 64 (w / 4) .. + 63, adds the bias and
// beta C.  Every mbarrier wait is bounded; a wait that gives up sets an error code (read with
// b2_nn_gemm_status), the CTA waits (bounded) for its issued products, frees its tensor memory
// and returns without storing.
#define T5_BM 128
#define T5_BN 128
#define T5_BK 64
#define T5_STAGE_BYTES ((T5_BM + T5_BN) * T5_BK * 2)
#define T5_SPIN (1 << 22)

__device__ int g_b2_nn_err = 0;

__device__ __forceinline__ uint32_t b2_nn_su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool b2_nn_mbar_wait(uint32_t a, uint32_t parity) {
  for (int it = 0; it < T5_SPIN; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ uint64_t b2_nn_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ uint32_t b2_nn_pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);     // .x = lo (low half), .y = hi
  return *reinterpret_cast<const uint32_t *>(&v);
}
// one operand tile (128 rows x 64 k) of a stage.  Thread unit = 8 consecutive k of one row
// (one 16-byte core-matrix row); lane = 8 a + b takes row 8 R + b and k chunk 4 KC + a, so a
// warp covers 8 rows x 4 chunks: with k contiguous in memory every row is read as 128
// contiguous bytes, with rows contiguous every k as 32 contiguous bytes, and each group of 8
// lanes stores 8 different 16-byte bank groups (no shared-memory conflicts).
__device__ __forceinline__ void b2_nn_fill(unsigned char *dst, int rows_valid, int k0, int K,
                                           const float *__restrict__ X, long long s_row, long long s_k,
                                           bool vec, int tid) {
#pragma unroll
  for (int u = 0; u < (128 * 8) / 256; ++u) {
    const int e = tid + 256 * u;
    const int r = 8 * ((e >> 5) & 15) + (e & 7), kc = 4 * (e >> 9) + ((e >> 3) & 3);
    const int gk0 = k0 + 8 * kc;
    float v[8];
    if (vec && r < rows_valid && gk0 + 8 <= K) {      // k contiguous and 16-byte aligned
      const float4 *src = reinterpret_cast<const float4 *>(X + (long long)r * s_row + gk0);
      const float4 x0 = src[0], x1 = src[1];
      v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w;
      v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
    } else {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int gk = gk0 + q;
        v[q] = (r < rows_valid && gk < K) ? X[(long long)r * s_row + (long long)gk * s_k] : 0.f;
      }
    }
    uint4 w;
    w.x = b2_nn_pack_bf16(v[0], v[1]);
    w.y = b2_nn_pack_bf16(v[2], v[3]);
    w.z = b2_nn_pack_bf16(v[4], v[5]);
    w.w = b2_nn_pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4 *>(dst + ((kc * 16 + (r >> 3)) * 128 + (r & 7) * 16)) = w;
  }
}

__global__ void __launch_bounds__(256)
k_nn_gemm_tc(int M, int N, int K, const float *__restrict__ A, long long sai, long long sak,
             const float *__restrict__ B, long long sbk, long long sbj, float *__restrict__ C,
             long long ldc, const float *__restrict__ bias, float beta) {
  extern __shared__ __align__(128) unsigned char t5_smem[];
  __shared__ __align__(8) unsigned long long sBar[2];
  __shared__ uint32_t sTmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i0 = blockIdx.y * T5_BM, j0 = blockIdx.x * T5_BN;
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(b2_nn_su32(&sBar[s])) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;"
                 :: "r"(b2_nn_su32(&sTmem)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tacc = sTmem;
  // instruction descriptor: f32 accumulator, bf16 A and B, both K-major, N = 128, M = 128
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(T5_BN >> 3) << 17) |
                         ((uint32_t)(T5_BM >> 4) << 24);
  const int mv = min(T5_BM, M - i0), nv = min(T5_BN, N - j0);
  const float *Ab = A + (long long)i0 * sai;
  const float *Bb = B + (long long)j0 * sbj;
  const int nk = (K + T5_BK - 1) / T5_BK;
  // 16-byte vector loads where k is contiguous and every row starts 16-byte aligned
  const bool vecA = sak == 1 && (sai & 3) == 0 && ((uintptr_t)Ab & 15) == 0;
  const bool vecB = sbk == 1 && (sbj & 3) == 0 && ((uintptr_t)Bb & 15) == 0;
  uint32_t ph = 0u, pend = 0u;          // per stage (bit s): mbarrier phase, product not yet seen complete
  bool fail = false;
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    unsigned char *sa = t5_smem + s * T5_STAGE_BYTES, *sb = sa + T5_BM * T5_BK * 2;
    if ((pend >> s) & 1u) {            // the product issued two steps ago read this stage
      if (b2_nn_mbar_wait(b2_nn_su32(&sBar[s]), (ph >> s) & 1u)) { ph ^= 1u << s; pend &= ~(1u << s); }
      else fail = true;
    }
    if (__syncthreads_or(fail)) break;
    b2_nn_fill(sa, mv, kt * T5_BK, K, Ab, sai, sak, vecA, tid);
    b2_nn_fill(sb, nv, kt * T5_BK, K, Bb, sbj, sbk, vecB, tid);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = b2_nn_su32(sa), b0 = b2_nn_su32(sb);
#pragma unroll
      for (int kk = 0; kk < T5_BK / 16; ++kk) {
        const uint64_t ad = b2_nn_sdesc(a0 + kk * 2 * 2048, 2048, 128);
        const uint64_t bd = b2_nn_sdesc(b0 + kk * 2 * 2048, 2048, 128);
        const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
            :: "r"(tacc), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(b2_nn_su32(&sBar[s])) : "memory");
    }
    pend |= 1u << s;
  }
  // wait for every issued product (the last one completes after all earlier ones)
#pragma unroll
  for (int s = 0; s < 2; ++s)
    if ((pend >> s) & 1u) {
      if (b2_nn_mbar_wait(b2_nn_su32(&sBar[s]), (ph >> s) & 1u)) { ph ^= 1u << s; pend &= ~(1u << s); }
      else fail = true;
    }
  if (fail && lane == 0) atomicExch(&g_b2_nn_err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  const bool any_fail = __syncthreads_or(fail);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!any_fail && nk > 0) {
    // tensor memory -> shared memory (row stride 65 floats: conflict-free both ways) -> C, one
    // 64-column half at a time, stored row by row (coalesced)
    float *stile = reinterpret_cast<float *>(t5_smem);
    const int r = 32 * (warp & 3) + lane;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      if ((warp >> 2) == h) {
#pragma unroll 1
        for (int cc = 0; cc < 64; cc += 16) {
          uint32_t v[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
              : "r"(tacc + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(64 * h + cc)));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int q = 0; q < 16; ++q) stile[r * 65 + cc + q] = __uint_as_float(v[q]);
        }
      }
      __syncthreads();
      for (int e = tid; e < T5_BM * 64; e += 256) {
        const int rr = e >> 6, c = e & 63;
        const int gi = i0 + rr, gj = j0 + 64 * h + c;
        if (gi < M && gj < N) {
          const float x = stile[rr * 65 + c] + (bias ? bias[gj] : 0.f);
          float *dst = C + (long long)gi * ldc + gj;
          *dst = beta != 0.f ? beta * *dst + x : x;
        }
      }
      __syncthreads();
    }
  } else if (!any_fail && nk == 0) {                  // K = 0: C = beta C + bias
    for (int e = tid; e < T5_BM * T5_BN; e += 256) {
      const int gi = i0 + e / T5_BN, gj = j0 + e % T5_BN;
      if (gi < M && gj < N) {
        float *dst = C + (long long)gi * ldc + gj;
        const float x = bias ? bias[gj] : 0.f;
        *dst = beta != 0.f ? beta * *dst + x : x;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" :: "r"(tacc) : "memory");
}

// column sums (bias gradients): out[j] (+)= sum_i X[i*ld + j]
__global__ void k_nn_colsum(int M, int N, const float *__restrict__ X, long long ld, float *__restrict__ out,
                            int accumulate) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  float s = 0.f;
  for (int i = 0; i < M; ++i) s += X[i * ld + j];
  out[j] = accumulate ? out[j] + s : s;
}

__global__ void k_nn_silu(long long n, const float *__restrict__ x, float *__restrict__ y) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { const float v = x[i]; y[i] = v / (1.f + expf(-v)); }
}

// dx = dy * silu'(x)
__global__ void k_nn_silu_bwd(long long n, const float *__restrict__ x, const float *__restrict__ dy,
                              float *__restrict__ dx) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float v = x[i], s = 1.f / (1.f + expf(-v));
    dx[i] = dy[i] * s * (1.f + v * (1.f - s));
  }
}

// radial basis: out[p][k] = exp(-g (r - mu_k)^2) fc(r), mu_k = rc k / (R-1)
__global__ void k_nn_rbf(long long P, int R, float rc, const float *__restrict__ r, float *__restrict__ out) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float rp = r[p];
  const float dmu = rc / (R - 1);
  const float g = 1.f / (2.f * dmu * dmu);
  const float fc = rp < rc ? 0.5f * (cospif(rp / rc) + 1.f) : 0.f;
  for (int k = 0; k < R; ++k) {
    const float d = rp - dmu * k;
    out[p * R + k] = expf(-g * d * d) * fc;
  }
}

// out[a][f] (+)= sum_{p in [ptr[a], ptr[a+1])} phi[p][f] * h[src[p]][f]   (one warp per atom)
__global__ void k_nn_message(int A, int F, const int *__restrict__ ptr, const int *__restrict__ src,
                             const float *__restrict__ phi, const float *__restrict__ h,
                             float *__restrict__ out, int accumulate) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (a >= A) return;
  for (int f = lane; f < F; f += 32) {
    float s = 0.f;
    for (int p = ptr[a]; p < ptr[a + 1]; ++p) s += phi[(long long)p * F + f] * h[(long long)src[p] * F + f];
    out[(long long)a * F + f] = accumulate ? out[(long long)a * F + f] + s : s;
  }
}

// dphi[p][f] = dm[dst[p]][f] * h[src[p]][f]
__global__ void k_nn_pairmul(long long P, int F, const int *__restrict__ src, const int *__restrict__ dst,
                             const float *__restrict__ dm, const float *__restrict__ h, float *__restrict__ out) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P * F) return;
  const long long p = e / F;
  const int f = (int)(e - p * F);
  out[e] = dm[(long long)dst[p] * F + f] * h[(long long)src[p] * F + f];
}

// x[p] = [h[a_p], h[b_p], rbf[p]]
__global__ void k_nn_gather(long long P, int F, int R, const int *__restrict__ pa, const int *__restrict__ pb,
                            const float *__restrict__ h, const float *__restrict__ rbf, float *__restrict__ x) {
  const int W = 2 * F + R;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P * W) return;
  const long long p = e / W;
  const int c = (int)(e - p * W);
  float v;
  if (c < F) v = h[(long long)pa[p] * F + c];
  else if (c < 2 * F) v = h[(long long)pb[p] * F + c - F];
  else v = rbf[p * R + c - 2 * F];
  x[e] = v;
}

// dh[a_p] += dx[p][0:F], dh[b_p] += dx[p][F:2F]
__global__ void k_nn_scatter(long long P, int F, int R, const int *__restrict__ pa, const int *__restrict__ pb,
                             const float *__restrict__ dx, float *__restrict__ dh) {
  const int W = 2 * F + R;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P * 2 * F) return;
  const long long p = e / (2 * F);
  const int c = (int)(e - p * 2 * F);
  const int atom = c < F ? pa[p] : pb[p];
  atomicAdd(&dh[(long long)atom * F + (c % F)], dx[p * W + c]);
}

__global__ void k_nn_embed(int A, int F, const int *__restrict__ type, const float *__restrict__ E,
                           float *__restrict__ h) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)A * F) return;
  const int a = (int)(e / F), f = (int)(e % F);
  h[e] = E[type[a] * F + f];
}

__global__ void k_nn_embed_bwd(int A, int F, const int *__restrict__ type, const float *__restrict__ dh,
                               float *__restrict__ dE) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)A * F) return;
  const int a = (int)(e / F), f = (int)(e % F);
  atomicAdd(&dE[type[a] * F + f], dh[e]);
}

// Assembly of the predicted density from the scalars (structure: oracle/nn_oracle.py visits()).
// Pair p (a<b, u = unit(R_b - R_a)): z[p][0..15]; site a: y[a][0..3].  The density is linear in
// the scalars, so one visitor enumerates (row, col, scalar index, coefficient) for the assembly
// (float64 atomic adds into a zeroed D) and for the gradient (dL/dz_k = sum coef * R[row, col]).
struct B2NnAtom { int mol, ao0, heavy, pad; };

template <typename Fn>
__device__ __forceinline__ void b2_nn_sym(int r, int c, int k, float coef, Fn &f) {
  f(r, c, k, coef);
  if (r != c) f(c, r, k, coef);
}

template <typename Fn>
__device__ void b2_nn_visit_pair(const B2NnAtom &A, const B2NnAtom &B, const float *u, Fn &f) {
  const int ns_a = A.heavy ? 2 : 1, ns_b = B.heavy ? 2 : 1;
  for (int i = 0; i < ns_a; ++i)
    for (int j = 0; j < ns_b; ++j) b2_nn_sym(A.ao0 + i, B.ao0 + j, 2 * i + j, 1.f, f);
  if (B.heavy)
    for (int i = 0; i < ns_a; ++i)
      for (int d = 0; d < 3; ++d) b2_nn_sym(A.ao0 + i, B.ao0 + 2 + d, 4 + i, u[d], f);
  if (A.heavy)
    for (int j = 0; j < ns_b; ++j)
      for (int c = 0; c < 3; ++c) b2_nn_sym(A.ao0 + 2 + c, B.ao0 + j, 6 + j, u[c], f);
  if (A.heavy && B.heavy)
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) {
        b2_nn_sym(A.ao0 + 2 + c, B.ao0 + 2 + d, 8, u[c] * u[d], f);
        b2_nn_sym(A.ao0 + 2 + c, B.ao0 + 2 + d, 9, (c == d ? 1.f : 0.f) - u[c] * u[d], f);
      }
  if (A.heavy) {
    for (int i = 0; i < 2; ++i)
      for (int c = 0; c < 3; ++c) b2_nn_sym(A.ao0 + i, A.ao0 + 2 + c, 10 + i, u[c], f);
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) f(A.ao0 + 2 + c, A.ao0 + 2 + d, 12, u[c] * u[d]);
  }
  if (B.heavy) {
    for (int j = 0; j < 2; ++j)
      for (int c = 0; c < 3; ++c) b2_nn_sym(B.ao0 + j, B.ao0 + 2 + c, 13 + j, -u[c], f);
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) f(B.ao0 + 2 + c, B.ao0 + 2 + d, 15, u[c] * u[d]);
  }
}

template <typename Fn>
__device__ void b2_nn_visit_site(const B2NnAtom &A, Fn &f) {
  const int o = A.ao0;
  f(o, o, 0, 1.f);
  if (A.heavy) {
    b2_nn_sym(o, o + 1, 1, 1.f, f);
    f(o + 1, o + 1, 2, 1.f);
    for (int c = 0; c < 3; ++c) f(o + 2 + c, o + 2 + c, 3, 1.f);
  }
}

__global__ void k_nn_assemble_pairs(long long P, const int *__restrict__ pa, const int *__restrict__ pb,
                                    const float *__restrict__ pu, const B2NnAtom *__restrict__ atoms,
                                    const long long *__restrict__ mat_off, const int *__restrict__ nao,
                                    const float *__restrict__ z, double *__restrict__ D,
                                    const double *__restrict__ Rg, float *__restrict__ dz) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const B2NnAtom A = atoms[pa[p]], B = atoms[pb[p]];
  const long long mo = mat_off[A.mol];
  const int n = nao[A.mol];
  const float u[3] = {pu[3 * p], pu[3 * p + 1], pu[3 * p + 2]};
  if (!Rg) {
    const float *zz = z + p * 16;
    auto put = [&](int r, int c, int k, float coef) { atomicAdd(&D[mo + (long long)r * n + c], (double)(coef * zz[k])); };
    b2_nn_visit_pair(A, B, u, put);
  } else {
    float g[16];
    for (int k = 0; k < 16; ++k) g[k] = 0.f;
    auto acc = [&](int r, int c, int k, float coef) { g[k] += coef * (float)Rg[mo + (long long)r * n + c]; };
    b2_nn_visit_pair(A, B, u, acc);
    for (int k = 0; k < 16; ++k) dz[p * 16 + k] = g[k];
  }
}

__global__ void k_nn_assemble_sites(int A_, const B2NnAtom *__restrict__ atoms, const long long *__restrict__ mat_off,
                                    const int *__restrict__ nao, const float *__restrict__ y, double *__restrict__ D,
                                    const double *__restrict__ Rg, float *__restrict__ dy) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= A_) return;
  const B2NnAtom A = atoms[a];
  const long long mo = mat_off[A.mol];
  const int n = nao[A.mol];
  if (!Rg) {
    const float *yy = y + (long long)a * 4;
    auto put = [&](int r, int c, int k, float coef) { atomicAdd(&D[mo + (long long)r * n + c], (double)(coef * yy[k])); };
    b2_nn_visit_site(A, put);
  } else {
    float g[4] = {0.f, 0.f, 0.f, 0.f};
    auto acc = [&](int r, int c, int k, float coef) { g[k] += coef * (float)Rg[mo + (long long)r * n + c]; };
    b2_nn_visit_site(A, acc);
    for (int k = 0; k < 4; ++k) dy[(long long)a * 4 + k] = g[k];
  }
}

// R = 2 (D - Dt) / n_entries over all entries; loss += sum (D - Dt)^2 / n_entries
__global__ void k_nn_residual(long long n, const double *__restrict__ D, const double *__restrict__ Dt,
                              double inv, double *__restrict__ R, double *__restrict__ loss) {
  __shared__ double red[8];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0;
  if (i < n) {
    const double r = D[i] - Dt[i];
    R[i] = 2.0 * r * inv;
    l = r * r * inv;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    atomicAdd(loss, s);
  }
}

// Adam: m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2; p -= lr mhat / (sqrt(vhat) + eps)
__global__ void k_nn_adam(long long n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                          float wd) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * p[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

static unsigned b2_blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

extern "C" {

int b2_nn_gemm(int M, int N, int K, const float *A, int64_t sai, int64_t sak, const float *B, int64_t sbk,
               int64_t sbj, float *C, int64_t ldc, const float *bias, float beta, int bf16, void *stream) {
  if (M < 0 || N < 0 || K < 0 || !A || !B || !C) return B2_ERR_ARG;
  if (M == 0 || N == 0) return B2_OK;
  if (bf16 == 2) {                       // tcgen05 tensor cores (bf16 inputs, fp32 accumulation)
    dim3 grid((N + T5_BN - 1) / T5_BN, (M + T5_BM - 1) / T5_BM);
    if (grid.y > 65535) return B2_ERR_SIZE;
    static bool attr[8] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 8) return B2_ERR_CUDA;
    if (!attr[dev]) {
      if (cudaFuncSetAttribute(k_nn_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * T5_STAGE_BYTES) !=
          cudaSuccess)
        return B2_ERR_CUDA;
      attr[dev] = true;
    }
    k_nn_gemm_tc<<<grid, 256, 2 * T5_STAGE_BYTES, (cudaStream_t)stream>>>(M, N, K, A, sai, sak, B, sbk, sbj, C,
                                                                          ldc, bias, beta);
    b2_count_launches(1);
    return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
  }
  dim3 grid((N + NN_BN - 1) / NN_BN, (M + NN_BM - 1) / NN_BM);
  if (grid.y > 65535) return B2_ERR_SIZE;
  k_nn_gemm<<<grid, 256, 0, (cudaStream_t)stream>>>(M, N, K, A, sai, sak, B, sbk, sbj, C, ldc, bias, beta, bf16);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_gemm_status(int reset, int *status) {
  if (!status) return B2_ERR_ARG;
  if (cudaMemcpyFromSymbol(status, g_b2_nn_err, sizeof(int)) != cudaSuccess) return B2_ERR_CUDA;
  if (reset) {
    const int z = 0;
    if (cudaMemcpyToSymbol(g_b2_nn_err, &z, sizeof(int)) != cudaSuccess) return B2_ERR_CUDA;
  }
  return B2_OK;
}

int b2_nn_colsum(int M, int N, const float *X, int64_t ld, float *out, int accumulate, void *stream) {
  if (N <= 0) return B2_OK;
  k_nn_colsum<<<b2_blocks(N, 128), 128, 0, (cudaStream_t)stream>>>(M, N, X, ld, out, accumulate);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_silu(int64_t n, const float *x, float *y, void *stream) {
  if (n <= 0) return B2_OK;
  k_nn_silu<<<b2_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(n, x, y);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_silu_bwd(int64_t n, const float *x, const float *dy, float *dx, void *stream) {
  if (n <= 0) return B2_OK;
  k_nn_silu_bwd<<<b2_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(n, x, dy, dx);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_rbf(int64_t P, int R, float rc, const float *r, float *out, void *stream) {
  if (P <= 0) return B2_OK;
  k_nn_rbf<<<b2_blocks(P, 128), 128, 0, (cudaStream_t)stream>>>(P, R, rc, r, out);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_message(int A, int F, const int *ptr, const int *src, const float *phi, const float *h, float *out,
                  int accumulate, void *stream) {
  if (A <= 0) return B2_OK;
  k_nn_message<<<b2_blocks((long long)A * 32, 256), 256, 0, (cudaStream_t)stream>>>(A, F, ptr, src, phi, h, out,
                                                                                    accumulate);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_pairmul(int64_t P, int F, const int *src, const int *dst, const float *dm, const float *h, float *out,
                  void *stream) {
  if (P <= 0) return B2_OK;
  k_nn_pairmul<<<b2_blocks(P * F, 256), 256, 0, (cudaStream_t)stream>>>(P, F, src, dst, dm, h, out);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_gather(int64_t P, int F, int R, const int *pa, const int *pb, const float *h, const float *rbf, float *x,
                 void *stream) {
  if (P <= 0) return B2_OK;
  k_nn_gather<<<b2_blocks(P * (2 * F + R), 256), 256, 0, (cudaStream_t)stream>>>(P, F, R, pa, pb, h, rbf, x);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_scatter(int64_t P, int F, int R, const int *pa, const int *pb, const float *dx, float *dh, void *stream) {
  if (P <= 0) return B2_OK;
  k_nn_scatter<<<b2_blocks(P * 2 * F, 256), 256, 0, (cudaStream_t)stream>>>(P, F, R, pa, pb, dx, dh);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_embed(int A, int F, const int *type, const float *E, float *h, void *stream) {
  if (A <= 0) return B2_OK;
  k_nn_embed<<<b2_blocks((long long)A * F, 256), 256, 0, (cudaStream_t)stream>>>(A, F, type, E, h);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_embed_bwd(int A, int F, const int *type, const float *dh, float *dE, void *stream) {
  if (A <= 0) return B2_OK;
  k_nn_embed_bwd<<<b2_blocks((long long)A * F, 256), 256, 0, (cudaStream_t)stream>>>(A, F, type, dh, dE);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

// D (zeroed by the caller) += predicted blocks.  With Dt: R (float64, n_mat) <- 2 (D - Dt)/n_mat,
// loss += mean squared error, dz / dy <- gradients of the loss w.r.t. the scalars.
int b2_nn_assemble(int64_t P, const int *pa, const int *pb, const float *pu, int A, const void *atoms,
                   const int64_t *mat_off, const int *nao, const float *z, const float *y, double *D,
                   int64_t n_mat, const double *Dt, double *R, float *dz, float *dy, double *loss, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const B2NnAtom *at = (const B2NnAtom *)atoms;
  const long long *mo = (const long long *)mat_off;
  if (A > 0) { k_nn_assemble_sites<<<b2_blocks(A, 128), 128, 0, st>>>(A, at, mo, nao, y, D, nullptr, nullptr); b2_count_launches(1); }
  if (P > 0) { k_nn_assemble_pairs<<<b2_blocks(P, 128), 128, 0, st>>>(P, pa, pb, pu, at, mo, nao, z, D, nullptr, nullptr); b2_count_launches(1); }
  if (Dt) {
    if (!R || !dz || !dy || !loss || n_mat <= 0) return B2_ERR_ARG;
    k_nn_residual<<<b2_blocks(n_mat, 256), 256, 0, st>>>(n_mat, D, Dt, 1.0 / (double)n_mat, R, loss);
    b2_count_launches(1);
    if (A > 0) { k_nn_assemble_sites<<<b2_blocks(A, 128), 128, 0, st>>>(A, at, mo, nao, y, D, R, dy); b2_count_launches(1); }
    if (P > 0) { k_nn_assemble_pairs<<<b2_blocks(P, 128), 128, 0, st>>>(P, pa, pb, pu, at, mo, nao, z, D, R, dz); b2_count_launches(1); }
  }
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

int b2_nn_adam(int64_t n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
               int step, float wd, void *stream) {
  if (n <= 0) return B2_OK;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_nn_adam<<<b2_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2, wd);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
}

}  // extern "C"
