// Exchange-correlation on the sm_100a tensor cores (tcgen05, accumulators in tensor memory).
//
// Same result as b2_xc_direct (exchange_correlation, nanoDFT.py:105-123; b3lyp.py:13-39) for
// float32: per tile of 128 grid points of one molecule
//   AO, dAO/dx,y,z for the tile          (CUDA cores; AO0 -> shared memory, AO1..3 -> TMEM)
//   X = AO0 D                             (tcgen05.mma kind::tf32, M=128 points, N=K=NB)
//   rho_c = sum_n X AO_c                  (CUDA cores, X read back from TMEM)
//   B3LYP per point                       (three parts on three of the point's threads)
//   Y = sum_c AO_c rt_c                   (CUDA cores -> shared memory)
//   V += AO0^T Y                          (tcgen05.mma, M=64 orbital rows, N=NB, K=128 points;
//                                          accumulated in TMEM across the CTA's tiles)
// NB = 16*Q is the molecule's orbital count padded to a multiple of 16 (Q = 1..5).
//
// Precision: both products use split TF32.  Each float32 operand x is split round-to-nearest
// into a TF32-exact head x1 and a float32 tail x - x1 (|tail| <= 2^-11 |x|); the D tail is
// rounded once more to TF32.  Three TF32 products per K step, A_h B_1 + A_h B_2 + A_l B_1,
// leave an error of ~2^-22 relative (the dropped A_l B_2 and the TF32 truncation of the
// tails), i.e. float32 quality.  AO values (including the approximate 2^x used for their
// primitives) do not depend on D: their errors are a fixed perturbation of the quadrature.
// Accumulation is float32 in TMEM.
//
// Shared-memory operand layouts (no swizzle, K-major; 8 x 16-byte "core matrices"):
//   * N tile (K = orbitals): AO0 for X = AO0 D, [orbital chunk n/4][point group p/8][p % 8]
//     [n % 4]; SBO 128 B between point groups, LBO 2048 B between orbital chunks.
//   * D: [k chunk][row group][row % 8][k % 4]; SBO 128 B, LBO (NB/8)*128 B.
//   * T tile (K = points): AO0^T and Y^T for V = AO0^T Y, [point chunk p/4][row group r/8]
//     [r % 8][p % 4]; SBO 128 B between row groups, LBO = (rows/8)*128 + 16 B between point
//     chunks (the extra 16 B staggers the chunks across shared-memory banks, so the 32 lanes
//     of a warp -- 32 consecutive points -- storing one orbital hit 32 different banks).
// Y^T reuses the N tile's bytes once X has been read back.
//
// Thread layout: 512 threads = 4 per grid point.  Warp w reads TMEM lanes 32*(w%4)..+31
// (the warp's lane quarter), so thread (qq = w/4, p = 32*(w%4)+lane) owns point p and the
// orbital quarter [qq*NB/4, (qq+1)*NB/4); B3LYP is split into Slater+B88, VWN and LYP parts
// on qq = 0, 1, 2.
//
// Every wait on an mbarrier is bounded; on timeout the kernel records an error code
// (read with b2_xc_tc_status), waits (bounded) for its issued MMAs, frees its TMEM and
// returns.
#include "device_plan.cuh"
#include "devmem.cuh"
#include "xc_math.cuh"
#include "xc.cuh"
#include <cstdint>

#define B2_XT_PT 128
#define B2_XT_NT 512
#define B2_XT_MAXSH 48
#define B2_XT_SPIN (1 << 20)

struct __align__(16) B2XtOrb {   // one atomic orbital of the CTA's molecule
  float e2[3], s;              // primitive exponents * log2(e); local shell (as float)
  float c[3], comp;            // coefficients (incl. angular factor); -1: s shell, 0..2: p_x,y,z
  float m2a[3], pad;           // -2 * exponent (radial derivative)
};

__device__ int g_b2_xt_err = 0;

__device__ __forceinline__ uint32_t b2_su32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// shared-memory matrix descriptor: start, leading / stride byte offsets, version 1, no swizzle
__device__ __forceinline__ uint64_t b2_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: float32 accumulator, TF32 A and B, A/B major, N, M
__device__ __forceinline__ uint32_t b2_idesc_tf32(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void b2_mma_tf32(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t idesc,
                                            uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :: "r"(dt), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
}
__device__ __forceinline__ void b2_mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(mbar) : "memory");
}
__device__ __forceinline__ void b2_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void b2_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void b2_fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void b2_mbar_init(uint32_t a, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool b2_mbar_wait(uint32_t a, uint32_t parity) {
  for (int it = 0; it < B2_XT_SPIN; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void b2_tmem_st4(uint32_t ta, float a, float b, float c, float d) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};"
               :: "r"(ta), "r"(__float_as_uint(a)), "r"(__float_as_uint(b)),
                  "r"(__float_as_uint(c)), "r"(__float_as_uint(d)) : "memory");
}
__device__ __forceinline__ float b2_ex2(float x) {     // 2^x (approximate; AO values only)
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ void b2_tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void b2_st4(float *p, float a, float b, float c, float d) {
  *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, d);
}
// element (point p, orbital n) of an N tile (floats)
__device__ __forceinline__ int b2_tile_idx(int p, int n) {
  return (((n >> 2) * 16 + (p >> 3)) * 8 + (p & 7)) * 4 + (n & 3);
}
// T tile with R rows: bytes between point chunks, and the float offset of (row r, chunk pc)
__host__ __device__ constexpr int b2_lt(int R) { return (R / 8) * 128 + 16; }
__device__ __forceinline__ int b2_tt_idx(int R, int r, int pc) {
  return (pc * b2_lt(R) + (r >> 3) * 128 + (r & 7) * 16) >> 2;
}

// named barrier of the 4 warps sharing TMEM lane quarter q (ids 1..4; 0 is __syncthreads)
__device__ __forceinline__ void b2_bar_quarter(int q) {
  asm volatile("bar.sync %0, 128;" :: "r"(q + 1) : "memory");
}
// 4-register TMEM load (this thread's lane, 4 consecutive columns)
__device__ __forceinline__ void b2_tmem_ld4(uint32_t ta, uint32_t *r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(ta));
}
__device__ __forceinline__ void b2_tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// round-to-nearest split into a TF32-exact head and a float32 tail
__device__ __forceinline__ void b2_split_rn(float x, float &hi, float &lo) {
  hi = __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
  lo = x - hi;
}

// Per-CTA body for NB = 16 Q.  sm: dynamic shared memory (floats), see b2_xt_smem_floats.
template <int Q>
__device__ void b2_xt_body(const B2MolDev &md, const B2XtOrb *sOrb, const double (*sR)[3],
                           float *sm, float *sRed, float *sFn, const double *__restrict__ coords,
                           const double *__restrict__ w, long long G, long long t0, int tpc,
                           const double *__restrict__ D, double *__restrict__ V, double &e_part,
                           uint32_t tbase, uint32_t mbar1, uint32_t mbar2, int *sAbort) {
  constexpr int NB = 16 * Q, OB = NB > 64 ? NB : 64;
  constexpr int R1 = (32 * b2_lt(NB)) / 4;          // floats of one N tile / Y^T tile
  constexpr int RT = (32 * b2_lt(OB)) / 4;          // floats of one AO0^T tile
  const int N = md.nao;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q4 = warp & 3, qq = warp >> 2, p = 32 * q4 + lane;
  float *sDh = sm, *sDl = sDh + NB * NB, *sAh = sDl + NB * NB, *sAl = sAh + R1;
  float *sTh = sAl + R1, *sTl = sTh + RT;
  float *sYh = sAh, *sYl = sAl;                     // Y^T tiles reuse the N tiles
  const uint32_t tl = tbase + ((uint32_t)(32 * q4) << 16);     // this warp's lane quarter
  const uint32_t colX = 0, colA = NB, colV = 4 * NB, colV2 = 5 * NB;
  const int nq0 = qq * 4 * Q;                       // first orbital of this thread's quarter

  // D (zero padded to NB) -> two round-to-nearest TF32 pieces, K-major core matrices; tiles
  // cleared (T-tile rows NB..63 are read as zero rows by the M=64 product)
  for (int e = tid; e < NB * NB; e += B2_XT_NT) {
    const int r = e / NB, k = e - r * NB;
    const float v = (r < N && k < N) ? (float)D[md.mat_off + (long long)r * N + k] : 0.f;
    float d1, d2, t;
    b2_split_rn(v, d1, t);
    d2 = __uint_as_float((__float_as_uint(t) + 0x1000u) & 0xFFFFE000u);
    const int idx = (((k >> 2) * (NB / 8) + (r >> 3)) * 8 + (r & 7)) * 4 + (k & 3);
    sDh[idx] = d1;
    sDl[idx] = d2;
  }
  for (int e = tid; e < 2 * R1 + 2 * RT; e += B2_XT_NT) sAh[e] = 0.f;
  b2_fence_async_smem();
  __syncthreads();

  const uint32_t id1 = b2_idesc_tf32(128, NB, 0, 0);   // X = AO0 D
  const uint32_t id2 = b2_idesc_tf32(64, NB, 0, 0);    // V = AO0^T Y (A = AO0^T, B = Y^T)
  uint32_t ph1 = 0, ph2 = 0;
  bool g2_pending = false, first = true;

  for (int tt = 0; tt < tpc; ++tt) {
    const long long g0 = (t0 + tt) * B2_XT_PT;
    if (g0 >= G) break;
    const int np = (int)min((long long)B2_XT_PT, G - g0);
    const bool valid = p < np;
    double px = 0, py = 0, pz = 0, wd = 0;
    if (valid) {
      px = coords[3 * (g0 + p)];
      py = coords[3 * (g0 + p) + 1];
      pz = coords[3 * (g0 + p) + 2];
      wd = w[g0 + p];
    }
    const float wp = (float)wd;
    // the previous tile's V product reads the T / Y^T tiles: wait before overwriting them
    if (g2_pending) {
      if (!b2_mbar_wait(mbar2, ph2)) { atomicExch(&g_b2_xt_err, 2); *sAbort = 1; }
      ph2 ^= 1;
      g2_pending = false;
      __syncthreads();
      if (*sAbort) return;
    }
    // ---- AO values of this thread's orbital quarter, 4 orbitals at a time
    int s_prev = -1;
    float dx = 0, dy = 0, dz = 0, ga = 0, gb = 0;
#pragma unroll 1
    for (int j4 = 0; j4 < Q; ++j4) {
      const int n0 = nq0 + 4 * j4;
      float a0[4], a1[4], a2[4], a3[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int n = n0 + u;
        a0[u] = a1[u] = a2[u] = a3[u] = 0.f;
        if (n < N && valid) {
          const float4 o0 = reinterpret_cast<const float4 *>(sOrb)[3 * n];
          const float4 o1 = reinterpret_cast<const float4 *>(sOrb)[3 * n + 1];
          const int sh = (int)o0.w;
          if (sh != s_prev) {          // same for every lane of the warp
            s_prev = sh;
            const float4 o2 = reinterpret_cast<const float4 *>(sOrb)[3 * n + 2];
            dx = (float)(px - sR[sh][0]);
            dy = (float)(py - sR[sh][1]);
            dz = (float)(pz - sR[sh][2]);
            const float r2 = dx * dx + dy * dy + dz * dz;
            const float ev0 = o1.x * b2_ex2(-o0.x * r2);
            const float ev1 = o1.y * b2_ex2(-o0.y * r2);
            const float ev2 = o1.z * b2_ex2(-o0.z * r2);
            ga = ev0 + ev1 + ev2;
            gb = o2.x * ev0 + o2.y * ev1 + o2.z * ev2;
          }
          const float comp = o1.w;
          if (comp < 0.f) {
            a0[u] = ga;
            a1[u] = gb * dx;
            a2[u] = gb * dy;
            a3[u] = gb * dz;
          } else {
            const float dc = comp == 0.f ? dx : (comp == 1.f ? dy : dz);
            const float t = dc * gb;
            a0[u] = dc * ga;
            a1[u] = (comp == 0.f ? ga : 0.f) + t * dx;
            a2[u] = (comp == 1.f ? ga : 0.f) + t * dy;
            a3[u] = (comp == 2.f ? ga : 0.f) + t * dz;
          }
        }
      }
      float hi[4], lo[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) b2_split_rn(a0[u], hi[u], lo[u]);
      b2_st4(sAh + b2_tile_idx(p, n0), hi[0], hi[1], hi[2], hi[3]);
      b2_st4(sAl + b2_tile_idx(p, n0), lo[0], lo[1], lo[2], lo[3]);
#pragma unroll
      for (int u = 0; u < 4; ++u) {                 // T tile: one float per orbital (conflict-free)
        const int it = b2_tt_idx(OB, n0 + u, p >> 2) + (p & 3);
        sTh[it] = hi[u];
        sTl[it] = lo[u];
      }
      b2_tmem_st4(tl + colA + n0, a1[0], a1[1], a1[2], a1[3]);
      b2_tmem_st4(tl + colA + NB + n0, a2[0], a2[1], a2[2], a2[3]);
      b2_tmem_st4(tl + colA + 2 * NB + n0, a3[0], a3[1], a3[2], a3[3]);
    }
    b2_tmem_wait_st();
    b2_fence_async_smem();
    b2_fence_before();
    __syncthreads();
    // ---- X = AO0 D = (A_h + A_l)(D_1 + D_2): four TF32 products per K step
    if (tid == 0) {
      b2_fence_after();
      const uint32_t aH = b2_su32(sAh), aL = b2_su32(sAl), dH = b2_su32(sDh), dL = b2_su32(sDl);
      constexpr uint32_t LBO_A = 2048, SBO_A = 128, LBO_D = (NB / 8) * 128, SBO_D = 128;
#pragma unroll 1
      for (int s = 0; s < NB / 8; ++s) {
        const uint64_t ah = b2_sdesc(aH + s * 2 * LBO_A, LBO_A, SBO_A);
        const uint64_t al = b2_sdesc(aL + s * 2 * LBO_A, LBO_A, SBO_A);
        const uint64_t bh = b2_sdesc(dH + s * 2 * LBO_D, LBO_D, SBO_D);
        const uint64_t bl = b2_sdesc(dL + s * 2 * LBO_D, LBO_D, SBO_D);
        b2_mma_tf32(tbase + colX, al, bh, id1, s > 0 ? 1u : 0u);
        b2_mma_tf32(tbase + colX, ah, bl, id1, 1u);
        b2_mma_tf32(tbase + colX, ah, bh, id1, 1u);
      }
      b2_mma_commit(mbar1);
    }
    if (!b2_mbar_wait(mbar1, ph1)) { atomicExch(&g_b2_xt_err, 1); *sAbort = 1; }
    ph1 ^= 1;
    b2_fence_after();
    // ---- rho partials over this thread's orbital quarter
    float r0 = 0.f, r1 = 0.f, r2 = 0.f, r3 = 0.f;
#pragma unroll 1
    for (int j4 = 0; j4 < Q; ++j4) {
      const int n0 = nq0 + 4 * j4;
      uint32_t x[4], b1[4], b2[4], b3[4];
      b2_tmem_ld4(tl + colX + n0, x);
      b2_tmem_ld4(tl + colA + n0, b1);
      b2_tmem_ld4(tl + colA + NB + n0, b2);
      b2_tmem_ld4(tl + colA + 2 * NB + n0, b3);
      const float4 ah = *reinterpret_cast<const float4 *>(sAh + b2_tile_idx(p, n0));
      const float4 al = *reinterpret_cast<const float4 *>(sAl + b2_tile_idx(p, n0));
      const float av[4] = {ah.x + al.x, ah.y + al.y, ah.z + al.z, ah.w + al.w};
      b2_tmem_wait_ld();
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float xv = __uint_as_float(x[u]);
        r0 += xv * av[u];
        r1 += xv * __uint_as_float(b1[u]);
        r2 += xv * __uint_as_float(b2[u]);
        r3 += xv * __uint_as_float(b3[u]);
      }
    }
    sRed[(qq * 4 + 0) * B2_XT_PT + p] = r0;
    sRed[(qq * 4 + 1) * B2_XT_PT + p] = r1;
    sRed[(qq * 4 + 2) * B2_XT_PT + p] = r2;
    sRed[(qq * 4 + 3) * B2_XT_PT + p] = r3;
    b2_fence_before();
    __syncthreads();
    if (*sAbort) return;
    float rho[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
      rho[c] = ((sRed[c * B2_XT_PT + p] + sRed[(4 + c) * B2_XT_PT + p]) + sRed[(8 + c) * B2_XT_PT + p]) +
               sRed[(12 + c) * B2_XT_PT + p];
    // ---- B3LYP in three parts: Slater + B88 (qq 0), VWN (qq 1), LYP (qq 2); the partial
    //      results reuse sRed once every thread has its rho
    __syncthreads();
    if (qq < 3) {
      const B2XcPoint<float> o = qq == 0 ? b2_b3lyp_x<float>(rho[0], rho[1], rho[2], rho[3])
                                 : qq == 1 ? b2_b3lyp_vwn<float>(rho[0], rho[1], rho[2], rho[3])
                                           : b2_b3lyp_lyp<float>(rho[0], rho[1], rho[2], rho[3]);
      sFn[(qq * 3 + 0) * B2_XT_PT + p] = o.exc;
      sFn[(qq * 3 + 1) * B2_XT_PT + p] = o.vrho;
      sFn[(qq * 3 + 2) * B2_XT_PT + p] = o.vgamma;
    }
    __syncthreads();
    const float exc = sFn[0 * B2_XT_PT + p] + (sFn[3 * B2_XT_PT + p] + sFn[6 * B2_XT_PT + p]);
    const float vrho = sFn[1 * B2_XT_PT + p] + (sFn[4 * B2_XT_PT + p] + sFn[7 * B2_XT_PT + p]);
    const float vg = sFn[2 * B2_XT_PT + p] + (sFn[5 * B2_XT_PT + p] + sFn[8 * B2_XT_PT + p]);
    if (qq == 0 && valid) e_part += (double)rho[0] * wd * (double)exc;
    const float rt0 = vrho * 0.5f * wp, f4 = 4.f * vg * wp;
    const float rt1 = f4 * rho[1], rt2 = f4 * rho[2], rt3 = f4 * rho[3];
    // ---- Y = AO0 rt0 + sum_c AO_c rt_c -> Y^T tiles (AO0 re-read from the T tile: the
    //      Y^T tiles overwrite the N tile)
#pragma unroll 1
    for (int j4 = 0; j4 < Q; ++j4) {
      const int n0 = nq0 + 4 * j4;
      uint32_t b1[4], b2[4], b3[4];
      b2_tmem_ld4(tl + colA + n0, b1);
      b2_tmem_ld4(tl + colA + NB + n0, b2);
      b2_tmem_ld4(tl + colA + 2 * NB + n0, b3);
      float av[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int it = b2_tt_idx(OB, n0 + u, p >> 2) + (p & 3);
        av[u] = sTh[it] + sTl[it];
      }
      b2_tmem_wait_ld();
      float y[4], yh[4], yl[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        y[u] = av[u] * rt0 + __uint_as_float(b1[u]) * rt1 + __uint_as_float(b2[u]) * rt2 +
               __uint_as_float(b3[u]) * rt3;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        b2_split_rn(y[u], yh[u], yl[u]);
        const int it = b2_tt_idx(NB, n0 + u, p >> 2) + (p & 3);
        sYh[it] = yh[u];
        sYl[it] = yl[u];
      }
    }
    b2_fence_async_smem();
    b2_fence_before();
    __syncthreads();
    // ---- V += AO0^T Y (M = 64 orbital rows; a second product covers rows 64..NB-1)
    if (tid == 0) {
      b2_fence_after();
      const uint32_t aH = b2_su32(sTh), aL = b2_su32(sTl), yH = b2_su32(sYh), yL = b2_su32(sYl);
      constexpr uint32_t LA = b2_lt(OB), LY = b2_lt(NB), SBO = 128;
      constexpr uint32_t off2 = (uint32_t)((NB > 64 ? (NB - 64) / 8 : 0) * 128);
#pragma unroll 1
      for (int s = 0; s < B2_XT_PT / 8; ++s) {
        const uint64_t ah = b2_sdesc(aH + 2 * s * LA, LA, SBO), al = b2_sdesc(aL + 2 * s * LA, LA, SBO);
        const uint64_t bh = b2_sdesc(yH + 2 * s * LY, LY, SBO), bl = b2_sdesc(yL + 2 * s * LY, LY, SBO);
        b2_mma_tf32(tbase + colV, al, bh, id2, (first && s == 0) ? 0u : 1u);
        b2_mma_tf32(tbase + colV, ah, bl, id2, 1u);
        b2_mma_tf32(tbase + colV, ah, bh, id2, 1u);
        if (NB > 64) {
          const uint64_t ah2 = b2_sdesc(aH + off2 + 2 * s * LA, LA, SBO);
          const uint64_t al2 = b2_sdesc(aL + off2 + 2 * s * LA, LA, SBO);
          b2_mma_tf32(tbase + colV2, al2, bh, id2, (first && s == 0) ? 0u : 1u);
          b2_mma_tf32(tbase + colV2, ah2, bl, id2, 1u);
          b2_mma_tf32(tbase + colV2, ah2, bh, id2, 1u);
        }
      }
      b2_mma_commit(mbar2);
    }
    g2_pending = true;
    first = false;
  }
  if (g2_pending) {
    if (!b2_mbar_wait(mbar2, ph2)) { atomicExch(&g_b2_xt_err, 3); *sAbort = 1; }
    __syncthreads();
    if (*sAbort) return;
  }
  if (first) return;                 // no tile processed
  b2_fence_after();
  // ---- V (M=64 layout: row 16*q4 + lane lives in lane 32*q4 + lane, lanes 0..15)
  const int mu = 16 * q4 + lane;
#pragma unroll 1
  for (int j4 = 0; j4 < Q; ++j4) {
    const int n0 = nq0 + 4 * j4;
    uint32_t v[4];
    b2_tmem_ld4(tl + colV + n0, v);
    b2_tmem_wait_ld();
    if (lane < 16 && mu < N) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float f = __uint_as_float(v[u]);
        if (n0 + u < N && f != 0.f) atomicAdd(&V[md.mat_off + (long long)mu * N + n0 + u], (double)f);
      }
    }
    if (NB > 64) {
      b2_tmem_ld4(tl + colV2 + n0, v);
      b2_tmem_wait_ld();
      const int mu2 = NB - 64 + mu;
      if (lane < 16 && mu2 >= 64 && mu2 < N) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float f = __uint_as_float(v[u]);
          if (n0 + u < N && f != 0.f) atomicAdd(&V[md.mat_off + (long long)mu2 * N + n0 + u], (double)f);
        }
      }
    }
  }
}

__host__ __device__ constexpr int b2_xt_smem_floats(int NB) {
  return 2 * NB * NB + 2 * (32 * b2_lt(NB)) / 4 + 2 * (32 * b2_lt(NB > 64 ? NB : 64)) / 4;
}

__global__ void __launch_bounds__(B2_XT_NT, 1)
k_xc_tc(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
        const long long *__restrict__ xblk_off, const long long *__restrict__ grid_off, int nmol,
        int tpc, const int *__restrict__ active, const double *__restrict__ coords,
        const double *__restrict__ w, const double *__restrict__ D, double *__restrict__ V,
        double *__restrict__ exc, const int *__restrict__ mol_map) {
  extern __shared__ __align__(128) float smem_f[];
  __shared__ B2XtOrb sOrb[80];
  __shared__ double sR[B2_XT_MAXSH][3];
  __shared__ float sRed[16 * B2_XT_PT];
  __shared__ double red[16];
  __shared__ __align__(8) unsigned long long sBar[2];
  __shared__ uint32_t sTmem;
  __shared__ int sAbort;
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (xblk_off[mid] <= (long long)blockIdx.x) lo = mid; else hi = mid - 1;
  }
  const int m = mol_map ? mol_map[lo] : lo;
  if (active && !active[m]) return;
  const B2MolDev md = mols[m];
  const int N = md.nao;
  const int Q = (N + 15) / 16, NB = 16 * Q;
  const int tid = threadIdx.x;
  // orbital table and shell centres
  for (int s = tid; s < md.nbas; s += B2_XT_NT) {
    const B2Shell &S = shells[md.sh_off + s];
    sR[s][0] = S.R[0];
    sR[s][1] = S.R[1];
    sR[s][2] = S.R[2];
    const int nc = S.l == 0 ? 1 : 3;
    for (int c = 0; c < nc; ++c) {
      B2XtOrb o;
      for (int k = 0; k < 3; ++k) {             // missing primitives: zero coefficient
        const bool has = k < S.nprim;
        o.e2[k] = has ? (float)(S.exp[k] * 1.4426950408889634) : 0.f;
        o.c[k] = has ? (float)S.coef[k] : 0.f;
        o.m2a[k] = has ? (float)(-2.0 * S.exp[k]) : 0.f;
      }
      o.s = (float)s;
      o.comp = S.l == 0 ? -1.f : (float)c;
      o.pad = 0.f;
      sOrb[S.ao0 + c] = o;
    }
  }
  if (tid == 0) {
    sAbort = 0;
    b2_mbar_init(b2_su32(&sBar[0]), 1);
    b2_mbar_init(b2_su32(&sBar[1]), 1);
  }
  // tensor memory: X (NB) + AO1..3 (3 NB) + V (NB, +NB for a second row block)
  const uint32_t need = (uint32_t)(NB > 64 ? 6 * NB : 5 * NB);
  const uint32_t ncols = need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
  if ((tid >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(b2_su32(&sTmem)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  b2_fence_before();
  __syncthreads();
  b2_fence_after();
  const uint32_t tbase = sTmem;
  const long long G = grid_off[m + 1] - grid_off[m];
  const long long t0 = (blockIdx.x - xblk_off[lo]) * (long long)tpc;
  const double *cm = coords + 3 * grid_off[m];
  const double *wm = w + grid_off[m];
  double e_part = 0;
  const uint32_t b1 = b2_su32(&sBar[0]), b2 = b2_su32(&sBar[1]);
  switch (Q) {
    case 1: b2_xt_body<1>(md, sOrb, sR, smem_f, sRed, sRed, cm, wm, G, t0, tpc, D, V, e_part, tbase, b1, b2, &sAbort); break;
    case 2: b2_xt_body<2>(md, sOrb, sR, smem_f, sRed, sRed, cm, wm, G, t0, tpc, D, V, e_part, tbase, b1, b2, &sAbort); break;
    case 3: b2_xt_body<3>(md, sOrb, sR, smem_f, sRed, sRed, cm, wm, G, t0, tpc, D, V, e_part, tbase, b1, b2, &sAbort); break;
    case 4: b2_xt_body<4>(md, sOrb, sR, smem_f, sRed, sRed, cm, wm, G, t0, tpc, D, V, e_part, tbase, b1, b2, &sAbort); break;
    default: b2_xt_body<5>(md, sOrb, sR, smem_f, sRed, sRed, cm, wm, G, t0, tpc, D, V, e_part, tbase, b1, b2, &sAbort); break;
  }
  // energy
  for (int o = 16; o > 0; o >>= 1) e_part += __shfl_down_sync(0xffffffffu, e_part, o);
  b2_fence_before();
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = e_part;
  __syncthreads();
  if (tid == 0) {
    double s = 0;
    for (int i = 0; i < B2_XT_NT / 32; ++i) s += red[i];
    if (!sAbort) atomicAdd(&exc[m], s);
  }
  b2_fence_after();
  if ((tid >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tbase), "r"(ncols) : "memory");
}

int b2_launch_xc_tc(const B2PlanDev &P, const int *active, const double *coords, const double *w,
                    const double *D, double *V, double *exc, cudaStream_t st) {
  const bool sub = P.sub.n > 0;
  const int nm = sub ? P.sub.n : P.h.nmol;
  const int *map = sub ? P.sub.mol_map : nullptr;
  const long long *xblk = sub ? P.sub.xtc : P.g.xblk_tc;
  const long long nblk = sub ? P.sub.n_xtc : P.g.n_xblk_tc;
  if (P.h.max_nbas > B2_XT_MAXSH || P.h.max_nao > 80) return B2_ERR_SIZE;
  if (!xblk) return B2_ERR_ARG;
  if (active) {
    int rc = b2_zero_active(P, active, V, nullptr, st);
    if (rc) return rc;
  } else {
    B2_CUDA_TRY(cudaMemsetAsync(V, 0, sizeof(double) * P.h.n_mat, st));
  }
  int rc = b2_zero_exc(P, active, exc, st);
  if (rc) return rc;
  const int NBmax = 16 * ((P.h.max_nao + 15) / 16);
  const size_t sm = sizeof(float) * (size_t)b2_xt_smem_floats(NBmax < 16 ? 16 : NBmax);
  B2_CUDA_TRY(cudaFuncSetAttribute(k_xc_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  if (nblk > 0) {
    k_xc_tc<<<(unsigned)nblk, B2_XT_NT, sm, st>>>(P.mols, P.shells, xblk, P.g.grid_off, nm,
                                                  P.g.tpc_tc, active, coords, w, D, V, exc, map);
    b2_count_launches(1);
  }
  return b2_sym_v(P, active, V, st);
}

// ============================================================================================
// Per-bucket persistent form (default).  Same products, precision and result as k_xc_tc, with
// these differences:
//   * one launch per orbital bucket (NB = 16 Q), shared memory and tensor memory sized for that
//     bucket (Q <= 2: two CTAs per SM);
//   * persistent CTAs pull work items (molecule, block of tiles) from a device queue (one
//     atomic counter per bucket, cleared before the launch) until it is empty; an item of an
//     inactive molecule is skipped;
//   * the radial factors ga = sum c e^{-a r^2} and gb = sum -2 a c e^{-a r^2} are evaluated once per
//     shell and tile (consecutive shells with the same centre and exponents, the 2s/2p pair of
//     STO-3G, share the exponentials); AO values go to the N and T tiles, AO gradients to tensor
//     memory (three columns per orbital) for the rho and Y phases;
//   * the next tile's grid point is loaded one tile ahead;
//   * the AO0^T tile holds NB rows: the M = 64 product's rows >= NB read whatever follows
//     (the next point chunk, or a pad), which only reaches accumulator rows >= NB, never read;
//   * 4 CTA barriers per tile (was 6): the AO evaluation and the tensor-memory stores of the AO
//     gradients run before the wait on the previous tile's V product.
// Tensor memory columns: X [0, NB), AO gradients [NB, 4NB), V [4NB, 5NB) (+ [5NB, 6NB) for
// NB > 64).
struct __align__(8) B2XtItem { int m, t0; };

// pad after each T tile: the M = 64 product reads (64 - NB) / 8 row groups past a chunk
template <int Q> __host__ __device__ constexpr int b2_xq_pad() { return 16 * Q < 64 ? 256 : 0; }
template <int Q>
__host__ __device__ constexpr int b2_xq_dyn_floats() {   // D, N / Y^T and T tiles, T pads
  return 2 * (16 * Q) * (16 * Q) + 4 * (32 * b2_lt(16 * Q)) / 4 + 2 * b2_xq_pad<Q>();
}
template <int Q> __host__ __device__ constexpr uint32_t b2_xq_tmem_cols() {
  return (16 * Q > 64 ? 6 : 5) * 16 * Q <= 64 ? 64 : (16 * Q > 64 ? 6 : 5) * 16 * Q <= 128 ? 128
         : (16 * Q > 64 ? 6 : 5) * 16 * Q <= 256 ? 256 : 512;
}

template <int Q>
__global__ void __launch_bounds__(B2_XT_NT, Q <= 2 ? 2 : 1)
k_xc_tq(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
        const B2XtItem *__restrict__ items, int n_items, int *__restrict__ queue,
        const long long *__restrict__ grid_off, int tpc, const int *__restrict__ active,
        const double *__restrict__ coords, const double *__restrict__ w, const double *__restrict__ D,
        double *__restrict__ V, double *__restrict__ exc) {
  constexpr int NB = 16 * Q;
  constexpr int R1 = (32 * b2_lt(NB)) / 4;          // floats of one N / Y^T / T tile
  constexpr uint32_t NCOL = b2_xq_tmem_cols<Q>();
  constexpr uint32_t colX = 0, colA = NB, colV = 4 * NB, colV2 = 5 * NB;
  extern __shared__ __align__(128) float smem_f[];
  __shared__ B2XtOrb sOrb[NB];
  __shared__ double sR[B2_XT_MAXSH][3];
  __shared__ float sRed[16 * B2_XT_PT];
  // NB = 80 leaves no room for a separate B3LYP exchange buffer: it reuses sRed (one more barrier)
  constexpr bool kAlias = Q >= 5;
  __shared__ float sFnArr[kAlias ? 1 : 9 * B2_XT_PT];
  float *sFn = kAlias ? sRed : sFnArr;
  __shared__ double red[16];
  __shared__ __align__(8) unsigned long long sBar[2];
  __shared__ uint32_t sTmem;
  __shared__ int sItem, sAbort;
  constexpr int PAD = b2_xq_pad<Q>();
  float *sDh = smem_f, *sDl = sDh + NB * NB, *sAh = sDl + NB * NB, *sAl = sAh + R1;
  float *sTh = sAl + R1, *sTl = sTh + R1 + PAD;     // each T tile followed by its pad
  float *sYh = sAh, *sYl = sAl;                     // Y^T tiles reuse the N tiles
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q4 = warp & 3, qq = warp >> 2, p = 32 * q4 + lane;
  const int nq0 = qq * 4 * Q;                       // first orbital of this thread's quarter

  if (tid == 0) {
    sAbort = 0;
    b2_mbar_init(b2_su32(&sBar[0]), 1);
    b2_mbar_init(b2_su32(&sBar[1]), 1);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(b2_su32(&sTmem)), "r"(NCOL) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // T tiles' pads: finite values (they only feed accumulator rows that are never read)
  for (int e = tid; e < PAD; e += B2_XT_NT) { sTh[R1 + e] = 0.f; sTl[R1 + e] = 0.f; }
  b2_fence_before();
  __syncthreads();
  b2_fence_after();
  const uint32_t tbase = sTmem;
  const uint32_t tl = tbase + ((uint32_t)(32 * q4) << 16);     // this warp's lane quarter
  const uint32_t mbar1 = b2_su32(&sBar[0]), mbar2 = b2_su32(&sBar[1]);
  const uint32_t id1 = b2_idesc_tf32(128, NB, 0, 0);            // X = AO0 D
  const uint32_t id2 = b2_idesc_tf32(64, NB, 0, 0);             // V = AO0^T Y
  uint32_t ph1 = 0, ph2 = 0;
  bool g2_pending = false, x_pending = false;      // an issued product not yet seen complete

  for (;;) {
    __syncthreads();                                // every thread is done with the last item
    if (tid == 0) sItem = atomicAdd(queue, 1);
    __syncthreads();
    const int it = sItem;
    if (it >= n_items || sAbort) break;
    const B2XtItem item = items[it];
    const int m = item.m;
    if (active && !active[m]) continue;             // uniform: every thread read the same item
    const B2MolDev md = mols[m];
    const int N = md.nao;
    const long long G = grid_off[m + 1] - grid_off[m];
    const double *cm = coords + 3 * grid_off[m];
    const double *wm = w + grid_off[m];
    // the previous item's V product may still read the T / Y^T tiles, and its V flush already
    // waited for it; here: orbital table, shell centres, D split into TF32 pieces
    for (int s = tid; s < md.nbas; s += B2_XT_NT) {
      const B2Shell &S = shells[md.sh_off + s];
      sR[s][0] = S.R[0];
      sR[s][1] = S.R[1];
      sR[s][2] = S.R[2];
      const int nc = S.l == 0 ? 1 : 3;
      bool same = false;                            // same centre and exponents as shell s-1
      if (s > 0) {
        const B2Shell &P0 = shells[md.sh_off + s - 1];
        same = P0.atom == S.atom && P0.nprim == S.nprim;
        for (int k = 0; k < S.nprim && same; ++k) same = P0.exp[k] == S.exp[k];
      }
      for (int c = 0; c < nc; ++c) {
        B2XtOrb o;
        for (int k = 0; k < 3; ++k) {
          const bool has = k < S.nprim;
          o.e2[k] = has ? (float)(S.exp[k] * 1.4426950408889634) : 0.f;
          o.c[k] = has ? (float)S.coef[k] : 0.f;
          o.m2a[k] = has ? (float)(-2.0 * S.exp[k]) : 0.f;
        }
        o.s = (float)s;
        o.comp = S.l == 0 ? -1.f : (float)c;
        o.pad = same ? 1.f : 0.f;
        sOrb[S.ao0 + c] = o;
      }
    }
    for (int e = tid; e < NB * NB; e += B2_XT_NT) {
      const int r = e / NB, k = e - r * NB;
      const float v = (r < N && k < N) ? (float)D[md.mat_off + (long long)r * N + k] : 0.f;
      float d1, d2, t;
      b2_split_rn(v, d1, t);
      d2 = __uint_as_float((__float_as_uint(t) + 0x1000u) & 0xFFFFE000u);
      const int idx = (((k >> 2) * (NB / 8) + (r >> 3)) * 8 + (r & 7)) * 4 + (k & 3);
      sDh[idx] = d1;
      sDl[idx] = d2;
    }
    // the orbital table and shell centres are read by every thread from the first tile on
    __syncthreads();
    double e_part = 0.0;
    bool first = true;
    // point of this thread in the next tile, loaded one tile ahead (the loads' latency overlaps
    // the current tile's work)
    double qx = 0, qy = 0, qz = 0, qw = 0;
    {
      const long long g1 = (long long)item.t0 * B2_XT_PT + p;
      if (g1 < G) { qx = cm[3 * g1]; qy = cm[3 * g1 + 1]; qz = cm[3 * g1 + 2]; qw = wm[g1]; }
    }
    for (int tt = 0; tt < tpc; ++tt) {
      const long long g0 = ((long long)item.t0 + tt) * B2_XT_PT;
      if (g0 >= G) break;
      const int np = (int)min((long long)B2_XT_PT, G - g0);
      const bool valid = p < np;
      const double px = qx, py = qy, pz = qz, wd = qw;     // zero for points past the grid
      {
        const long long g1 = g0 + B2_XT_PT + p;
        qx = qy = qz = qw = 0.0;
        if (tt + 1 < tpc && g1 < G) { qx = cm[3 * g1]; qy = cm[3 * g1 + 1]; qz = cm[3 * g1 + 2]; qw = wm[g1]; }
      }
      const float wp = (float)wd;
      // ---- AO values (registers) and AO gradients (tensor memory) of this thread's orbitals
      float a0[4 * Q];
      {
        int s_prev = -1;
        float ev0 = 0, ev1 = 0, ev2 = 0, dx = 0, dy = 0, dz = 0, ga = 0, gb = 0;
#pragma unroll
        for (int j4 = 0; j4 < Q; ++j4) {
          float a1[4], a2[4], a3[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int n = nq0 + 4 * j4 + u;
            float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
            if (n < N && valid) {
              const float4 o0 = reinterpret_cast<const float4 *>(sOrb)[3 * n];
              const float4 o1 = reinterpret_cast<const float4 *>(sOrb)[3 * n + 1];
              const int sh = min(max((int)o0.w, 0), B2_XT_MAXSH - 1);   // table index (clamped)
              if (sh != s_prev) {        // same for every lane of the warp
                const float4 o2 = reinterpret_cast<const float4 *>(sOrb)[3 * n + 2];
                if (!(o2.w != 0.f && sh == s_prev + 1 && s_prev >= 0)) {
                  dx = (float)(px - sR[sh][0]);
                  dy = (float)(py - sR[sh][1]);
                  dz = (float)(pz - sR[sh][2]);
                  const float r2 = dx * dx + dy * dy + dz * dz;
                  ev0 = b2_ex2(-o0.x * r2);
                  ev1 = b2_ex2(-o0.y * r2);
                  ev2 = b2_ex2(-o0.z * r2);
                }
                s_prev = sh;
                ga = o1.x * ev0 + o1.y * ev1 + o1.z * ev2;
                gb = o2.x * o1.x * ev0 + o2.y * o1.y * ev1 + o2.z * o1.z * ev2;
              }
              const float comp = o1.w;
              if (comp < 0.f) {          // s:   AO = ga, grad AO = gb d
                v0 = ga;
                v1 = gb * dx;
                v2 = gb * dy;
                v3 = gb * dz;
              } else {                   // p_k: AO = d_k ga, grad AO = ga e_k + d_k gb d
                const float dk = comp == 0.f ? dx : (comp == 1.f ? dy : dz);
                const float t = dk * gb;
                v0 = dk * ga;
                v1 = (comp == 0.f ? ga : 0.f) + t * dx;
                v2 = (comp == 1.f ? ga : 0.f) + t * dy;
                v3 = (comp == 2.f ? ga : 0.f) + t * dz;
              }
            }
            a0[4 * j4 + u] = v0;
            a1[u] = v1;
            a2[u] = v2;
            a3[u] = v3;
          }
          b2_tmem_st4(tl + colA + nq0 + 4 * j4, a1[0], a1[1], a1[2], a1[3]);
          b2_tmem_st4(tl + colA + NB + nq0 + 4 * j4, a2[0], a2[1], a2[2], a2[3]);
          b2_tmem_st4(tl + colA + 2 * NB + nq0 + 4 * j4, a3[0], a3[1], a3[2], a3[3]);
        }
      }
      // the previous tile's V product reads the T / Y^T tiles: wait before overwriting them.
      // A wait that gives up is combined over the CTA at the next CTA barrier, so every thread
      // leaves at the same point.
      bool fail = false;
      if (g2_pending) {
        if (b2_mbar_wait(mbar2, ph2)) { ph2 ^= 1; g2_pending = false; }
        else { atomicExch(&g_b2_xt_err, 2); fail = true; }
      }
#pragma unroll
      for (int j4 = 0; j4 < Q; ++j4) {
        const int n0 = nq0 + 4 * j4;
        float hi[4], lo[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) b2_split_rn(a0[4 * j4 + u], hi[u], lo[u]);
        b2_st4(sAh + b2_tile_idx(p, n0), hi[0], hi[1], hi[2], hi[3]);
        b2_st4(sAl + b2_tile_idx(p, n0), lo[0], lo[1], lo[2], lo[3]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {               // T tile: one float per orbital (conflict-free)
          const int ti = b2_tt_idx(NB, n0 + u, p >> 2) + (p & 3);
          sTh[ti] = hi[u];
          sTl[ti] = lo[u];
        }
      }
      b2_tmem_wait_st();
      b2_fence_async_smem();
      b2_fence_before();
      if (__syncthreads_or(fail)) { sAbort = 1; break; }            // [1]
      x_pending = true;
      // ---- X = AO0 D = (A_h + A_l)(D_1 + D_2): three TF32 products per K step
      if (tid == 0) {
        b2_fence_after();
        const uint32_t aH = b2_su32(sAh), aL = b2_su32(sAl), dH = b2_su32(sDh), dL = b2_su32(sDl);
        constexpr uint32_t LBO_A = 2048, SBO_A = 128, LBO_D = (NB / 8) * 128, SBO_D = 128;
#pragma unroll 1
        for (int s = 0; s < NB / 8; ++s) {
          const uint64_t ah = b2_sdesc(aH + s * 2 * LBO_A, LBO_A, SBO_A);
          const uint64_t al = b2_sdesc(aL + s * 2 * LBO_A, LBO_A, SBO_A);
          const uint64_t bh = b2_sdesc(dH + s * 2 * LBO_D, LBO_D, SBO_D);
          const uint64_t bl = b2_sdesc(dL + s * 2 * LBO_D, LBO_D, SBO_D);
          b2_mma_tf32(tbase + colX, al, bh, id1, s > 0 ? 1u : 0u);
          b2_mma_tf32(tbase + colX, ah, bl, id1, 1u);
          b2_mma_tf32(tbase + colX, ah, bh, id1, 1u);
        }
        b2_mma_commit(mbar1);
      }
      // ---- rho partials over this thread's orbitals: X and the AO gradients from tensor memory
      //      (every load waited with nothing in between: the destination registers are written
      //      asynchronously), AO values from registers
      if (b2_mbar_wait(mbar1, ph1)) { ph1 ^= 1; x_pending = false; }
      else { atomicExch(&g_b2_xt_err, 1); fail = true; }
      b2_fence_after();
      float r0 = 0.f, r1 = 0.f, r2 = 0.f, r3 = 0.f;
#pragma unroll
      for (int j4 = 0; j4 < Q; ++j4) {
        const int n0 = nq0 + 4 * j4;
        uint32_t x[4], b1[4], b2[4], b3[4];
        b2_tmem_ld4(tl + colX + n0, x);
        b2_tmem_ld4(tl + colA + n0, b1);
        b2_tmem_ld4(tl + colA + NB + n0, b2);
        b2_tmem_ld4(tl + colA + 2 * NB + n0, b3);
        b2_tmem_wait_ld();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float xv = __uint_as_float(x[u]);
          r0 += xv * a0[4 * j4 + u];
          r1 += xv * __uint_as_float(b1[u]);
          r2 += xv * __uint_as_float(b2[u]);
          r3 += xv * __uint_as_float(b3[u]);
        }
      }
      sRed[(qq * 4 + 0) * B2_XT_PT + p] = r0;
      sRed[(qq * 4 + 1) * B2_XT_PT + p] = r1;
      sRed[(qq * 4 + 2) * B2_XT_PT + p] = r2;
      sRed[(qq * 4 + 3) * B2_XT_PT + p] = r3;
      // from here to the V product a point's four threads (warps q4, q4+4, q4+8, q4+12) exchange
      // data only among themselves through sRed / sFn entries of their own points: a barrier per
      // lane quarter (128 threads) instead of the whole CTA.  The N tile is no longer read (the AO
      // values come from registers), so a quarter may start writing Y^T over it.
      b2_bar_quarter(q4);                                           // [2]
      float rho[4];
#pragma unroll
      for (int c = 0; c < 4; ++c)
        rho[c] = ((sRed[c * B2_XT_PT + p] + sRed[(4 + c) * B2_XT_PT + p]) + sRed[(8 + c) * B2_XT_PT + p]) +
                 sRed[(12 + c) * B2_XT_PT + p];
      if (kAlias) b2_bar_quarter(q4);                               // sFn overwrites sRed
      // ---- B3LYP in three parts: Slater + B88 (qq 0), VWN (qq 1), LYP (qq 2)
      if (qq < 3) {
        const B2XcPoint<float> o = qq == 0 ? b2_b3lyp_x<float>(rho[0], rho[1], rho[2], rho[3])
                                   : qq == 1 ? b2_b3lyp_vwn<float>(rho[0], rho[1], rho[2], rho[3])
                                             : b2_b3lyp_lyp<float>(rho[0], rho[1], rho[2], rho[3]);
        sFn[(qq * 3 + 0) * B2_XT_PT + p] = o.exc;
        sFn[(qq * 3 + 1) * B2_XT_PT + p] = o.vrho;
        sFn[(qq * 3 + 2) * B2_XT_PT + p] = o.vgamma;
      }
      b2_bar_quarter(q4);                                           // [3]
      const float ex = sFn[0 * B2_XT_PT + p] + (sFn[3 * B2_XT_PT + p] + sFn[6 * B2_XT_PT + p]);
      const float vrho = sFn[1 * B2_XT_PT + p] + (sFn[4 * B2_XT_PT + p] + sFn[7 * B2_XT_PT + p]);
      const float vg = sFn[2 * B2_XT_PT + p] + (sFn[5 * B2_XT_PT + p] + sFn[8 * B2_XT_PT + p]);
      if (qq == 0 && valid) e_part += (double)rho[0] * wd * (double)ex;
      const float rt0 = vrho * 0.5f * wp, f4 = 4.f * vg * wp;
      const float rt1 = f4 * rho[1], rt2 = f4 * rho[2], rt3 = f4 * rho[3];
      // ---- Y_n = AO_n rt0 + grad AO_n . rt -> Y^T tiles (AO values from registers; the Y^T
      //      tiles overwrite the N tile, which the X product has finished reading)
#pragma unroll
      for (int j4 = 0; j4 < Q; ++j4) {
        const int n0 = nq0 + 4 * j4;
        uint32_t b1[4], b2[4], b3[4];
        b2_tmem_ld4(tl + colA + n0, b1);
        b2_tmem_ld4(tl + colA + NB + n0, b2);
        b2_tmem_ld4(tl + colA + 2 * NB + n0, b3);
        b2_tmem_wait_ld();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float y = a0[4 * j4 + u] * rt0 + __uint_as_float(b1[u]) * rt1 + __uint_as_float(b2[u]) * rt2 +
                          __uint_as_float(b3[u]) * rt3;
          float yh, yl;
          b2_split_rn(y, yh, yl);
          const int ti = b2_tt_idx(NB, n0 + u, p >> 2) + (p & 3);
          sYh[ti] = yh;
          sYl[ti] = yl;
        }
      }
      b2_fence_async_smem();
      b2_fence_before();
      if (__syncthreads_or(fail)) { sAbort = 1; break; }            // [4]
      // ---- V += AO0^T Y (M = 64 orbital rows; a second product covers rows 64..NB-1)
      if (tid == 0) {
        b2_fence_after();
        const uint32_t aH = b2_su32(sTh), aL = b2_su32(sTl), yH = b2_su32(sYh), yL = b2_su32(sYl);
        constexpr uint32_t LA = b2_lt(NB), SBO = 128;
        constexpr uint32_t off2 = (uint32_t)((NB > 64 ? (NB - 64) / 8 : 0) * 128);
#pragma unroll 1
        for (int s = 0; s < B2_XT_PT / 8; ++s) {
          const uint64_t ah = b2_sdesc(aH + 2 * s * LA, LA, SBO), al = b2_sdesc(aL + 2 * s * LA, LA, SBO);
          const uint64_t bh = b2_sdesc(yH + 2 * s * LA, LA, SBO), bl = b2_sdesc(yL + 2 * s * LA, LA, SBO);
          b2_mma_tf32(tbase + colV, al, bh, id2, (first && s == 0) ? 0u : 1u);
          b2_mma_tf32(tbase + colV, ah, bl, id2, 1u);
          b2_mma_tf32(tbase + colV, ah, bh, id2, 1u);
          if (NB > 64) {
            const uint64_t ah2 = b2_sdesc(aH + off2 + 2 * s * LA, LA, SBO);
            const uint64_t al2 = b2_sdesc(aL + off2 + 2 * s * LA, LA, SBO);
            b2_mma_tf32(tbase + colV2, al2, bh, id2, (first && s == 0) ? 0u : 1u);
            b2_mma_tf32(tbase + colV2, ah2, bl, id2, 1u);
            b2_mma_tf32(tbase + colV2, ah2, bh, id2, 1u);
          }
        }
        b2_mma_commit(mbar2);
      }
      g2_pending = true;
      first = false;
    }
    // ---- end of the item: wait for its last V product, flush V and the energy
    if (g2_pending && !sAbort) {
      if (b2_mbar_wait(mbar2, ph2)) { ph2 ^= 1; g2_pending = false; }
      else { atomicExch(&g_b2_xt_err, 3); sAbort = 1; }
    }
    __syncthreads();
    if (sAbort) break;
    if (!first) {
      b2_fence_after();
      const int mu = 16 * q4 + lane;               // M=64 layout: row 16 q4 + lane in lanes 0..15
#pragma unroll 1
      for (int j4 = 0; j4 < Q; ++j4) {
        const int n0 = nq0 + 4 * j4;
        uint32_t v[4];
        b2_tmem_ld4(tl + colV + n0, v);
        b2_tmem_wait_ld();
        if (lane < 16 && mu < N) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float f = __uint_as_float(v[u]);
            if (n0 + u < N && f != 0.f) atomicAdd(&V[md.mat_off + (long long)mu * N + n0 + u], (double)f);
          }
        }
        if (NB > 64) {
          b2_tmem_ld4(tl + colV2 + n0, v);
          b2_tmem_wait_ld();
          const int mu2 = NB - 64 + mu;
          if (lane < 16 && mu2 >= 64 && mu2 < N) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const float f = __uint_as_float(v[u]);
              if (n0 + u < N && f != 0.f) atomicAdd(&V[md.mat_off + (long long)mu2 * N + n0 + u], (double)f);
            }
          }
        }
      }
      for (int o = 16; o > 0; o >>= 1) e_part += __shfl_down_sync(0xffffffffu, e_part, o);
      if (lane == 0) red[warp] = e_part;
      b2_fence_before();
      __syncthreads();
      if (tid == 0) {
        double sum = 0;
        for (int i = 0; i < B2_XT_NT / 32; ++i) sum += red[i];
        atomicAdd(&exc[m], sum);
      }
    }
  }
  // leaving: a product may still be in flight only after an abort; wait for it (bounded)
  if (x_pending) b2_mbar_wait(mbar1, ph1);
  if (g2_pending) b2_mbar_wait(mbar2, ph2);
  b2_fence_before();
  __syncthreads();
  b2_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tbase), "r"(NCOL) : "memory");
}

template <int Q>
static int b2_xq_launch(const B2PlanDev &P, const B2XtItem *items, int n_items, int *queue,
                        const int *active, const double *coords, const double *w, const double *D,
                        double *V, double *exc, cudaStream_t st) {
  const size_t sm = sizeof(float) * (size_t)b2_xq_dyn_floats<Q>();
  static int occ[8] = {0};                      // CTAs per SM (per device, filled on first use)
  int dev = 0;
  B2_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 8) return B2_ERR_CUDA;
  if (!occ[dev]) {
    B2_CUDA_TRY(cudaFuncSetAttribute(k_xc_tq<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int o = 0, nsm = 0;
    B2_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_xc_tq<Q>, B2_XT_NT, sm));
    B2_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    occ[dev] = std::max(1, o) * nsm;
  }
  const int grid = std::min(n_items, occ[dev]);
  const int tpc = P.g.xq_tpc[Q - 1] > 0 ? P.g.xq_tpc[Q - 1] : std::max(1, P.g.tpc_tc);
  k_xc_tq<Q><<<grid, B2_XT_NT, sm, st>>>(P.mols, P.shells, items, n_items, queue, P.g.grid_off,
                                          tpc, active, coords, w, D, V, exc);
  return B2_OK;
}

int b2_launch_xc_tq(const B2PlanDev &P, const int *active, const double *coords, const double *w,
                    const double *D, double *V, double *exc, cudaStream_t st) {
  const bool sub = P.sub.n > 0;
  const B2XtItem *items = (const B2XtItem *)(sub ? P.sub.xq_items : P.g.xq_items);
  const std::vector<long long> &off = sub ? P.sub.xq_off_h : P.g.xq_off_h;
  if (P.h.max_nbas > B2_XT_MAXSH || P.h.max_nao > 80) return B2_ERR_SIZE;
  if (!items || off.size() != B2_NBKT + 1 || !P.g.xq_queue) return B2_ERR_ARG;
  if (active) {
    int rc = b2_zero_active(P, active, V, nullptr, st);
    if (rc) return rc;
  } else {
    B2_CUDA_TRY(cudaMemsetAsync(V, 0, sizeof(double) * P.h.n_mat, st));
  }
  int rc = b2_zero_exc(P, active, exc, st);
  if (rc) return rc;
  B2_CUDA_TRY(cudaMemsetAsync(P.g.xq_queue, 0, sizeof(int) * B2_NBKT, st));
  // one launch per bucket on the plan's bucket streams (forked from / joined to `st`)
  B2_CUDA_TRY(cudaEventRecord(P.bkt_ev[B2_NBKT], st));
  for (int b = B2_NBKT - 1; b >= 0; --b) {
    const int n = (int)(off[b + 1] - off[b]);
    if (n <= 0) continue;
    cudaStream_t s = P.bkt_stream[b];
    B2_CUDA_TRY(cudaStreamWaitEvent(s, P.bkt_ev[B2_NBKT], 0));
    const B2XtItem *it = items + off[b];
    int *q = P.g.xq_queue + b;
    switch (b) {
      case 0: rc = b2_xq_launch<1>(P, it, n, q, active, coords, w, D, V, exc, s); break;
      case 1: rc = b2_xq_launch<2>(P, it, n, q, active, coords, w, D, V, exc, s); break;
      case 2: rc = b2_xq_launch<3>(P, it, n, q, active, coords, w, D, V, exc, s); break;
      case 3: rc = b2_xq_launch<4>(P, it, n, q, active, coords, w, D, V, exc, s); break;
      default: rc = b2_xq_launch<5>(P, it, n, q, active, coords, w, D, V, exc, s); break;
    }
    if (rc) return rc;
    b2_count_launches(1);
    B2_CUDA_TRY(cudaGetLastError());
    B2_CUDA_TRY(cudaEventRecord(P.bkt_ev[b], s));
    B2_CUDA_TRY(cudaStreamWaitEvent(st, P.bkt_ev[b], 0));
  }
  return b2_sym_v(P, active, V, st);
}

// work items (molecule, first tile) of the per-bucket kernel for the molecules `mols`, grouped
// by orbital bucket (off: B2_NBKT + 1 bucket starts), `tpc` tiles per item
static void b2_xq_items(const B2PlanDev &P, const std::vector<int> &mols, int tpc, std::vector<B2XtItem> &items,
                        std::vector<long long> &off) {
  off.assign(B2_NBKT + 1, 0);
  std::vector<std::vector<B2XtItem>> per(B2_NBKT);
  for (int m : mols) {
    const int b = std::min(B2_NBKT - 1, (P.h.mols[m].nao - 1) / 16);
    const long long nt = (P.g.grid_off_h[m + 1] - P.g.grid_off_h[m] + B2_XT_PT - 1) / B2_XT_PT;
    const int tb = P.g.xq_tpc[b] > 0 ? P.g.xq_tpc[b] : tpc;
    for (long long t = 0; t < nt; t += tb) per[b].push_back(B2XtItem{m, (int)t});
  }
  items.clear();
  for (int b = 0; b < B2_NBKT; ++b) {
    items.insert(items.end(), per[b].begin(), per[b].end());
    off[b + 1] = (long long)items.size();
  }
}

int b2_xc_tc_status_read(int reset) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_b2_xt_err, sizeof(int)) != cudaSuccess) return -1;
  if (reset) {
    const int z = 0;
    cudaMemcpyToSymbol(g_b2_xt_err, &z, sizeof(int));
  }
  return v;
}

int b2_xq_build(const B2PlanDev &P, const std::vector<int> &mols, void **items, std::vector<long long> &off) {
  std::vector<B2XtItem> it;
  b2_xq_items(P, mols, std::max(1, P.g.tpc_tc), it, off);
  B2XtItem *d = nullptr;
  B2_CUDA_TRY(b2_dmalloc_t(&d, sizeof(B2XtItem) * std::max<size_t>(1, it.size())));
  if (!it.empty())
    B2_CUDA_TRY(cudaMemcpy(d, it.data(), sizeof(B2XtItem) * it.size(), cudaMemcpyHostToDevice));
  b2_dfree(*items);
  *items = d;
  return B2_OK;
}
