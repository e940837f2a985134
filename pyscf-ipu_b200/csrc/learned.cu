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

// Tensor-core form of the same product: bf16 inputs, fp32 accumulation, mma.sync m16n8k16.
// CTA tile 128x128, 8 warps (2 x 4), each warp 64 x 32 (4 x 4 fragments); K step 32.
// Fragment layout (PTX ISA, mma.m16n8k16 .bf16): g = lane/4, t = lane%4;
//   A regs: (g, 2t..2t+1), (g+8, 2t..), (g, 2t+8..), (g+8, 2t+8..)     B regs: (k=2t.., n=g), (k=2t+8.., n=g)
//   C: (g, 2t..2t+1), (g+8, 2t..2t+1)
#define TC_BM 128
#define TC_BN 128
#define TC_BK 32
#define TC_LD (TC_BK + 8)

__global__ void __launch_bounds__(256)
k_nn_gemm_tc(int M, int N, int K, const float *__restrict__ A, long long sai, long long sak,
             const float *__restrict__ B, long long sbk, long long sbj, float *__restrict__ C,
             long long ldc, const float *__restrict__ bias, float beta) {
  __shared__ __align__(16) __nv_bfloat16 As[TC_BM][TC_LD];   // [m][k]
  __shared__ __align__(16) __nv_bfloat16 Bs[TC_BN][TC_LD];   // [n][k]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;                     // 2 x 4 warps
  const int g = lane >> 2, t = lane & 3;
  const int i0 = blockIdx.y * TC_BM, j0 = blockIdx.x * TC_BN;
  float acc[4][4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
  for (int k0 = 0; k0 < K; k0 += TC_BK) {
    for (int e = threadIdx.x; e < TC_BM * TC_BK; e += 256) {
      const int ii = e / TC_BK, kk = e % TC_BK;
      const int gi = i0 + ii, gk = k0 + kk;
      As[ii][kk] = __float2bfloat16_rn((gi < M && gk < K) ? A[gi * sai + gk * sak] : 0.f);
    }
    for (int e = threadIdx.x; e < TC_BN * TC_BK; e += 256) {
      const int jj = e % TC_BN, kk = e / TC_BN;
      const int gj = j0 + jj, gk = k0 + kk;
      Bs[jj][kk] = __float2bfloat16_rn((gj < N && gk < K) ? B[gk * sbk + gj * sbj] : 0.f);
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < TC_BK; ks += 16) {
      unsigned af[4][4], bfr[4][2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int r = wm * 64 + mt * 16 + g;
        af[mt][0] = *reinterpret_cast<const unsigned *>(&As[r][ks + 2 * t]);
        af[mt][1] = *reinterpret_cast<const unsigned *>(&As[r + 8][ks + 2 * t]);
        af[mt][2] = *reinterpret_cast<const unsigned *>(&As[r][ks + 2 * t + 8]);
        af[mt][3] = *reinterpret_cast<const unsigned *>(&As[r + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int cidx = wn * 32 + nt * 8 + g;
        bfr[nt][0] = *reinterpret_cast<const unsigned *>(&Bs[cidx][ks + 2 * t]);
        bfr[nt][1] = *reinterpret_cast<const unsigned *>(&Bs[cidx][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
              "{%0,%1,%2,%3};\n"
              : "+f"(acc[mt][nt][0]), "+f"(acc[mt][nt][1]), "+f"(acc[mt][nt][2]), "+f"(acc[mt][nt][3])
              : "r"(af[mt][0]), "r"(af[mt][1]), "r"(af[mt][2]), "r"(af[mt][3]), "r"(bfr[nt][0]), "r"(bfr[nt][1]));
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int gi = i0 + wm * 64 + mt * 16 + g + 8 * h;
          const int gj = j0 + wn * 32 + nt * 8 + 2 * t + q;
          if (gi < M && gj < N) {
            const float v = acc[mt][nt][2 * h + q] + (bias ? bias[gj] : 0.f);
            float *dst = C + gi * ldc + gj;
            *dst = beta != 0.f ? beta * *dst + v : v;
          }
        }
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
  if (bf16 == 2) {                       // tensor cores (bf16 inputs, fp32 accumulation)
    dim3 grid((N + TC_BN - 1) / TC_BN, (M + TC_BM - 1) / TC_BM);
    if (grid.y > 65535) return B2_ERR_SIZE;
    k_nn_gemm_tc<<<grid, 256, 0, (cudaStream_t)stream>>>(M, N, K, A, sai, sak, B, sbk, sbj, C, ldc, bias, beta);
    b2_count_launches(1);
    return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
  }
  dim3 grid((N + NN_BN - 1) / NN_BN, (M + NN_BM - 1) / NN_BM);
  if (grid.y > 65535) return B2_ERR_SIZE;
  k_nn_gemm<<<grid, 256, 0, (cudaStream_t)stream>>>(M, N, K, A, sai, sak, B, sbk, sbj, C, ldc, bias, beta, bf16);
  b2_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? B2_OK : B2_ERR_CUDA;
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
