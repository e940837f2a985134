// Nuclear gradients of converged RKS SCFs on the GPU, batched over a plan's molecules: the
// reference's grad(mol, coords, weight, mo_coeff, mo_energy) = grad_elec + grad_nuc
// (nanoDFT.py:403-477), which builds int2e_ip1 / int1e_ip* on the host and contracts them with
// einsums.  Here every term is contracted as it is generated, in float64:
//
//   k_grad_dm   dm0 = 2 C_occ C_occ^T, dme0 = 2 C_occ eps_occ C_occ^T (nanoDFT.py:405-406);
//   k_grad_2e   d/dR of 1/2 <D, J> - hyb/4 <D, K> (the vj / vk terms, nanoDFT.py:416-418): one
//               warp per task of the ERI work list (bra shell pair x up to 32 kets of one
//               class), one canonical shell quartet per lane, class-specialised;
//   k_grad_1e   d/dR of <D, T + V_nuc> - <dme0, S> (h1aos and s1, nanoDFT.py:420-424): one CTA
//               per molecule, one ordered shell pair per thread;
//   k_grad_xc   d/dR of E_xc at fixed density and grid (V_xc, nanoDFT.py:408-415): one CTA per
//               32 grid points of one molecule, AO values, D-products and B3LYP staged in
//               shared memory;
//   k_grad_nuc  nuclear repulsion (grad_nuc, nanoDFT.py:428-438).
//
// The per-term math is grad_math.cuh, the same code the host-check build tests against the
// finite-difference oracle.
#include <algorithm>
#include <utility>
#include <vector>
#include "device_plan.cuh"
#include "devmem.cuh"
#include "grad_math.cuh"

#define B2G_TP 32                  // grid points per XC tile (one warp's lanes)
#define B2G_XC_THREADS 256

__global__ void __launch_bounds__(256)
k_grad_dm(const B2MolDev *__restrict__ mols, const double *__restrict__ C, const double *__restrict__ eps,
          double *__restrict__ D, double *__restrict__ W) {
  const int m = blockIdx.x;
  const B2MolDev md = mols[m];
  const int N = md.nao, NN = N * N;
  const double *Cm = C + md.mat_off;
  const double *em = eps + (long long)m * B2_MAXNAO;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    double s = 0, t = 0;
    for (int k = 0; k < md.nocc; ++k) {
      const double p = Cm[a * N + k] * Cm[b * N + k];
      s += p;
      t += p * em[k];
    }
    D[md.mat_off + e] = 2.0 * s;
    W[md.mat_off + e] = 2.0 * t;
  }
}

// Two-electron part over canonical shell quartets: one warp per task of the float32 ERI work
// list (bra shell pair IJ x up to 32 kets of one class, the group G fixing all four angular
// momenta); the warp takes the task's canonical kets (KL <= IJ; the list also holds kets KL > IJ
// of the bra's last shell, which the s8 writer needs) one after the other and shares the work
// of each shell quartet over its lanes:
//   * primitive pairs: the bra's (once per task) and the ket's (once per quartet) Gaussian
//     products, one pair per lane, into shared memory; pairs with |K| < 1e-20 (coefficients
//     included) are dropped;
//   * primitive quartets in batches of 32, one per lane: the quartet's scalars (W - P, W - Q,
//     the recursion factors, pref x Boys F_0..F_L) into shared memory;
//   * per primitive quartet of the batch, the lanes split the Obara-Saika vertical recursion
//     for [e0|f0]^(m) level by level (one buffer per warp; the recursion steps of the class --
//     target, sources, direction, factors -- are tabulated once per CTA), once with the bra
//     raised by one (the bra-centre derivatives) and once with the ket raised by one (the
//     derivative on the centre of K); the weighted sums over primitives (1, 2 alpha, 2 beta;
//     1, 2 gamma) stay in the registers of the lane that owns the (e, f) entry;
//   * the horizontal recursion and the contraction with the symmetrised Gamma run with the
//     quartet's components spread over the lanes; the derivatives on the centres of K and L
//     (the latter by translation invariance) are reduced over the warp per quartet, the bra
//     centres' once per task.
// Same formulas as the serial b2g_canonical_quartet (grad_math.cuh), which the host build runs.
// v[e][f][m] of NCB primitive quartets at once (buffer c at v + c NV; v[0][0][m] already set),
// lanes over (step, quartet) pairs level by level.  Quartet c's scalars: cs + c B2G_CS (W - P,
// W - Q, rho/zeta, rho/eta, 1/(2 zeta), 1/(2 eta), 1/(2 (zeta + eta))) and its pair records
// (P - A from the bra's, Q - C from the ket's), selected by idx[c].
template <typename S, int LE, int LF, int NCB>
__device__ __forceinline__ void b2g_vrr_warp(double *v, const B2gOp *ops, int lane, int nv, const double *cs,
                                             const double *bpr, const double *kpr, const unsigned char (*idx)[2]);
#define B2G_PP 12                  // doubles per primitive-pair record
#define B2G_CS 18                  // doubles per primitive-quartet record
#define B2G_KTHR 1e-20             // primitive pairs with |K| below this are dropped

template <typename S, int LE, int LF, int NCB>
__device__ __forceinline__ void b2g_vrr_warp(double *v, const B2gOp *ops, int lane, int nv, const double *cs,
                                             const double *bpr, const double *kpr, const unsigned char (*idx)[2]) {
#pragma unroll
  for (int l1 = 1; l1 <= LE; ++l1) {
    const int lo = b2g_cstart(l1) - 1, n = (b2g_cstart(l1 + 1) - 1 - lo) * NCB;
    for (int t = lane; t < n; t += 32) {
      const int o = lo + t / NCB, c = t - (t / NCB) * NCB;
      if (c >= nv) continue;
      const B2gOp op = ops[o];
      const double *q = cs + c * B2G_CS, *B = bpr + idx[c][0] * B2G_PP;
      const double x = B[6 + op.dd], y = q[op.dd];
      const double cc = (double)op.c1 * q[8], rb = q[6];
      double *vc = v + c * S::NV;
#pragma unroll
      for (int m = 0; m < S::SM; ++m)              // independent in m: unrolled, predicated
        if (m <= op.mmax) {
          double u = x * vc[op.s1 + m] + y * vc[op.s1 + m + 1];
          if (op.s2 >= 0) u += cc * (vc[op.s2 + m] - rb * vc[op.s2 + m + 1]);
          vc[op.dst + m] = u;
        }
    }
    __syncwarp();
  }
#pragma unroll
  for (int l2 = 1; l2 <= LF; ++l2) {
    const int lo = S::NOB + (b2g_cstart(l2) - 1) * S::NE;
    const int n = (b2g_cstart(l2 + 1) - b2g_cstart(l2)) * S::NE * NCB;
    for (int t = lane; t < n; t += 32) {
      const int o = lo + t / NCB, c = t - (t / NCB) * NCB;
      if (c >= nv) continue;
      const B2gOp op = ops[o];
      if (op.mmax < 0) continue;
      const double *q = cs + c * B2G_CS, *K = kpr + idx[c][1] * B2G_PP;
      const double x = K[6 + op.dd], y = q[3 + op.dd];
      const double cc = (double)op.c1 * q[9], rk = q[7], c3 = (double)op.c3 * q[10];
      double *vc = v + c * S::NV;
#pragma unroll
      for (int m = 0; m < S::SM; ++m)
        if (m <= op.mmax) {
          double u = x * vc[op.s1 + m] + y * vc[op.s1 + m + 1];
          if (op.s2 >= 0) u += cc * (vc[op.s2 + m] - rk * vc[op.s2 + m + 1]);
          if (op.s3 >= 0) u += c3 * vc[op.s3 + m + 1];
          vc[op.dst + m] = u;
        }
    }
    __syncwarp();
  }
}

// per-class sizes of the two-electron kernel's shared memory (doubles per warp)
template <int G> struct B2g2e {
  static constexpr int LA = b2g_group_l(G, 0), LB = b2g_group_l(G, 1), LC = b2g_group_l(G, 2),
                       LD = b2g_group_l(G, 3);
  static constexpr int L = LA + LB + LC + LD + 1;
  using SB = B2gVrr<LA + LB + 1, LC + LD, L>;              // bra raised by one
  using SK = B2gVrr<LA + LB, LC + LD + 1, L>;              // ket raised by one
  static constexpr int NVB = SB::NV > SK::NV ? SB::NV : SK::NV;
  static constexpr int NACC = 3 * SB::NACC + 2 * SK::NACC;
  // primitive quartets whose recursions run side by side (buffers of at most 1200 doubles)
  static constexpr int NCB = 1200 / NVB >= 4 ? 4 : (1200 / NVB >= 2 ? 2 : 1);
  static constexpr int NBUF = NCB * NVB > NACC ? NCB * NVB : NACC;
  static constexpr int PER_WARP = NBUF + 2 * B2_MAXPRIM * B2_MAXPRIM * B2G_PP + 32 * B2G_CS;
  static constexpr size_t SMEM = sizeof(double) * 4 * PER_WARP;
};

// primitive pair (p, q) of shells (s, t): exponents, zeta, P, P - R_s, K (coefficients
// included), 1 / zeta
__device__ __forceinline__ void b2g_pair_rec(const B2Shell &s, const B2Shell &t, int p, int q, double R2,
                                             double *o) {
  const double al = s.exp[p], be = t.exp[q], z = al + be, iz = 1.0 / z;
  o[0] = al;
  o[1] = be;
  o[2] = z;
  for (int x = 0; x < 3; ++x) {
    const double P = (al * s.R[x] + be * t.R[x]) * iz;
    o[3 + x] = P;
    o[6 + x] = P - s.R[x];
  }
  o[9] = exp(-al * be * iz * R2) * s.coef[p] * t.coef[q];
  o[10] = iz;
  o[11] = 0.0;
}

// lanes 0..np-1 each form one primitive pair; the surviving ones are packed into rec; returns
// their number (same value on every lane)
__device__ __forceinline__ int b2g_pairs_warp(const B2Shell &s, const B2Shell &t, double R2, double *rec, int lane) {
  const int np = s.nprim * t.nprim;
  double o[B2G_PP];
  bool keep = false;
  if (lane < np) {
    b2g_pair_rec(s, t, lane / t.nprim, lane - (lane / t.nprim) * t.nprim, R2, o);
    keep = fabs(o[9]) >= B2G_KTHR;
  }
  const unsigned bal = __ballot_sync(0xffffffffu, keep);
  if (keep) {
    const int pos = __popc(bal & ((1u << lane) - 1u));
#pragma unroll
    for (int k = 0; k < B2G_PP; ++k) rec[pos * B2G_PP + k] = o[k];
  }
  __syncwarp();
  return __popc(bal);
}

template <int G>
__global__ void __launch_bounds__(128)
k_grad_2e(const B2EriTask *__restrict__ tasks, long long ntask, const B2MolDev *__restrict__ mols,
          const B2PairInfo *__restrict__ pinfo, const int *__restrict__ cls_list,
          const B2Shell *__restrict__ shells, const double *__restrict__ btab, const double *__restrict__ D,
          double hyb, double *__restrict__ grad) {
  using C2 = B2g2e<G>;
  constexpr int LA = C2::LA, LB = C2::LB, LC = C2::LC, LD = C2::LD, L = C2::L;
  constexpr int na = 2 * LA + 1, nb = 2 * LB + 1, nc = 2 * LC + 1, nd = 2 * LD + 1, NCMP = na * nb * nc * nd;
  using SB = typename C2::SB;
  using SK = typename C2::SK;
  constexpr int KB = (SB::NACC + 31) / 32, KK = (SK::NACC + 31) / 32;
  extern __shared__ __align__(16) double g2_smem[];
  __shared__ B2gOp sopB[SB::NOP], sopK[SK::NOP];
  __shared__ unsigned char sIdx[4][32][2];
  for (int o = threadIdx.x; o < SB::NOP; o += blockDim.x) sopB[o] = SB::op(o);
  for (int o = threadIdx.x; o < SK::NOP; o += blockDim.x) sopK[o] = SK::op(o);
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ti = (long long)blockIdx.x * 4 + w;
  if (ti >= ntask) return;                        // whole warp (no CTA barrier follows)
  double *v = g2_smem + (size_t)w * C2::PER_WARP;
  double *bpr = v + C2::NBUF, *kpr = bpr + B2_MAXPRIM * B2_MAXPRIM * B2G_PP;
  double *cs = kpr + B2_MAXPRIM * B2_MAXPRIM * B2G_PP;
  const B2EriTask tk = tasks[ti];
  const B2MolDev md = mols[tk.mol];
  const B2PairInfo bp = pinfo[md.sp_off + tk.IJ];
  const B2Shell &a = shells[md.sh_off + bp.I], &b = shells[md.sh_off + bp.J];
  const double *Dm = D + md.mat_off;
  const int N = md.nao;
  double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};   // this lane's part of the bra-centre sums
  double AB[3], AB2 = 0;
  for (int x = 0; x < 3; ++x) { AB[x] = a.R[x] - b.R[x]; AB2 += AB[x] * AB[x]; }
  const int nbp = b2g_pairs_warp(a, b, AB2, bpr, lane);
  double *gm = grad + 3ll * md.atm_off;
  for (int kq = 0; kq < tk.count; ++kq) {
    const int KL = cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + kq];
    if (KL > tk.IJ) continue;                     // uniform over the warp
    const B2PairInfo kp = pinfo[md.sp_off + KL];
    const B2Shell &c = shells[md.sh_off + kp.I], &d = shells[md.sh_off + kp.J];
    double CD[3], CD2 = 0;
    for (int x = 0; x < 3; ++x) { CD[x] = c.R[x] - d.R[x]; CD2 += CD[x] * CD[x]; }
    const int nkp = b2g_pairs_warp(c, d, CD2, kpr, lane);
    double accB[3][KB], accK[2][KK];
#pragma unroll
    for (int k = 0; k < KB; ++k) accB[0][k] = accB[1][k] = accB[2][k] = 0.0;
#pragma unroll
    for (int k = 0; k < KK; ++k) accK[0][k] = accK[1][k] = 0.0;
    const int ncombo = nbp * nkp;
    for (int c0 = 0; c0 < ncombo; c0 += 32) {
      // ---- scalars of up to 32 primitive quartets, one per lane
      const int cb = c0 + lane;
      if (cb < ncombo) {
        const int ib = cb / nkp, ik = cb - (cb / nkp) * nkp;
        const double *B = bpr + ib * B2G_PP, *K = kpr + ik * B2G_PP;
        const double z = B[2], e = K[2], iz = B[10], ie = K[10];
        const double rs = rsqrt(z + e), inv = rs * rs;          // 1/sqrt(zeta+eta), 1/(zeta+eta)
        double *o = cs + lane * B2G_CS;
        double PQ2 = 0;
        for (int x = 0; x < 3; ++x) {
          const double P = B[3 + x], Q = K[3 + x];
          const double W = (z * P + e * Q) * inv;
          o[x] = W - P;                             // WP
          o[3 + x] = W - Q;                         // WQ
          PQ2 += (P - Q) * (P - Q);
        }
        const double rho = z * e * inv;
        const double pref = 34.98683665524972 * iz * ie * rs * B[9] * K[9];   // 2 pi^(5/2) / (z e sqrt(z+e)) K K
        double F[L + 1];
        b2_boys<double, L, double>(rho * PQ2, btab, F);
        o[6] = e * inv;                           // rho / zeta
        o[7] = z * inv;                           // rho / eta
        o[8] = 0.5 * iz;
        o[9] = 0.5 * ie;
        o[10] = 0.5 * inv;
#pragma unroll
        for (int m = 0; m <= L; ++m) o[11 + m] = pref * F[m];
        sIdx[w][lane][0] = (unsigned char)ib;
        sIdx[w][lane][1] = (unsigned char)ik;
      }
      __syncwarp();
      const int nq = min(32, ncombo - c0);
      constexpr int NCB = C2::NCB;
      for (int q0 = 0; q0 < nq; q0 += NCB) {
        const int nv = min(NCB, nq - q0);
        const double *csq = cs + q0 * B2G_CS;
        // bra raised: [e0|f0], e <= LA + LB + 1, f <= LC + LD
        for (int t = lane; t < nv * (L + 1); t += 32) {
          const int c = t / (L + 1), m = t - (t / (L + 1)) * (L + 1);
          v[c * SB::NV + m] = csq[c * B2G_CS + 11 + m];
        }
        __syncwarp();
        b2g_vrr_warp<SB, LA + LB + 1, LC + LD, NCB>(v, sopB, lane, nv, csq, bpr, kpr, sIdx[w] + q0);
#pragma unroll
        for (int k = 0; k < KB; ++k) {
          const int t = lane + 32 * k;
          if (t < SB::NACC) {
            const int ie = t / SB::NF, jf = t - (t / SB::NF) * SB::NF;
            for (int c = 0; c < nv; ++c) {
              const double x = v[c * SB::NV + ie * SB::SE + jf * SB::SM];
              const double *B = bpr + sIdx[w][q0 + c][0] * B2G_PP;
              accB[0][k] += x;
              accB[1][k] += 2.0 * B[0] * x;
              accB[2][k] += 2.0 * B[1] * x;
            }
          }
        }
        __syncwarp();
        // ket raised: e <= LA + LB, f <= LC + LD + 1
        for (int t = lane; t < nv * (L + 1); t += 32) {
          const int c = t / (L + 1), m = t - (t / (L + 1)) * (L + 1);
          v[c * SK::NV + m] = csq[c * B2G_CS + 11 + m];
        }
        __syncwarp();
        b2g_vrr_warp<SK, LA + LB, LC + LD + 1, NCB>(v, sopK, lane, nv, csq, bpr, kpr, sIdx[w] + q0);
#pragma unroll
        for (int k = 0; k < KK; ++k) {
          const int t = lane + 32 * k;
          if (t < SK::NACC) {
            const int ie = t / SK::NF, jf = t - (t / SK::NF) * SK::NF;
            for (int c = 0; c < nv; ++c) {
              const double x = v[c * SK::NV + ie * SK::SE + jf * SK::SM];
              const double *K = kpr + sIdx[w][q0 + c][1] * B2G_PP;
              accK[0][k] += x;
              accK[1][k] += 2.0 * K[0] * x;
            }
          }
        }
        __syncwarp();
      }
    }
    // weighted sums to shared memory: accB[w][e][f], then accK[w][e][f]
#pragma unroll
    for (int k = 0; k < KB; ++k) {
      const int t = lane + 32 * k;
      if (t < SB::NACC)
        for (int q = 0; q < 3; ++q) v[q * SB::NACC + t] = accB[q][k];
    }
#pragma unroll
    for (int k = 0; k < KK; ++k) {
      const int t = lane + 32 * k;
      if (t < SK::NACC)
        for (int q = 0; q < 2; ++q) v[3 * SB::NACC + q * SK::NACC + t] = accK[q][k];
    }
    __syncwarp();
    const auto *aB = reinterpret_cast<const double (*)[SB::NE][SB::NF]>(v);
    const auto *aK = reinterpret_cast<const double (*)[SK::NE][SK::NF]>(v + 3 * SB::NACC);
    const double deg = (bp.I == bp.J ? 1.0 : 2.0) * (kp.I == kp.J ? 1.0 : 2.0) * (KL == tk.IJ ? 1.0 : 2.0);
    double gC[3] = {0, 0, 0}, g3[3] = {0, 0, 0};
    for (int cmp = lane; cmp < NCMP; cmp += 32) {
      const int id = cmp % nd, ic = (cmp / nd) % nc, ib = (cmp / (nd * nc)) % nb, ia = cmp / (nd * nc * nb);
      const int i = a.ao0 + ia, j = b.ao0 + ib, k = c.ao0 + ic, l = d.ao0 + id;
      const double gmv = deg * (0.5 * Dm[i * N + j] * Dm[k * N + l] -
                                0.125 * hyb * (Dm[i * N + l] * Dm[j * N + k] + Dm[i * N + k] * Dm[j * N + l]));
      if (gmv == 0.0) continue;
      int ea[3], eb[3], ec[3], ed[3];
      b2g_comp(LA, ia, ea); b2g_comp(LB, ib, eb); b2g_comp(LC, ic, ec); b2g_comp(LD, id, ed);
      for (int x = 0; x < 3; ++x) {
        int up[3], dn[3];
        for (int q = 0; q < 3; ++q) { up[q] = ea[q] + (q == x); dn[q] = ea[q] - (q == x); }
        double dA = b2g_hrr(aB, 1, up, eb, ec, ed, AB, CD);
        if (ea[x]) dA -= (double)ea[x] * b2g_hrr(aB, 0, dn, eb, ec, ed, AB, CD);
        for (int q = 0; q < 3; ++q) { up[q] = eb[q] + (q == x); dn[q] = eb[q] - (q == x); }
        double dB = b2g_hrr(aB, 2, ea, up, ec, ed, AB, CD);
        if (eb[x]) dB -= (double)eb[x] * b2g_hrr(aB, 0, ea, dn, ec, ed, AB, CD);
        for (int q = 0; q < 3; ++q) { up[q] = ec[q] + (q == x); dn[q] = ec[q] - (q == x); }
        double dC = b2g_hrr(aK, 1, ea, eb, up, ed, AB, CD);
        if (ec[x]) dC -= (double)ec[x] * b2g_hrr(aK, 0, ea, eb, dn, ed, AB, CD);
        gA[x] += gmv * dA;
        gB[x] += gmv * dB;
        gC[x] += gmv * dC;
        g3[x] -= gmv * (dA + dB + dC);
      }
    }
    for (int x = 0; x < 3; ++x) {
      double u = gC[x], t = g3[x];
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        u += __shfl_xor_sync(0xffffffffu, u, o);
        t += __shfl_xor_sync(0xffffffffu, t, o);
      }
      if (lane == 0) {
        atomicAdd(gm + 3 * c.atom + x, u);
        atomicAdd(gm + 3 * d.atom + x, t);
      }
    }
    __syncwarp();                                 // v and the pair records are rewritten next
  }
  // the bra centres are the warp's: one sum over the lanes, one atomic per component
  for (int x = 0; x < 3; ++x) {
    double u = gA[x], t = gB[x];
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      u += __shfl_xor_sync(0xffffffffu, u, o);
      t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    if (lane == 0) {
      atomicAdd(gm + 3 * a.atom + x, u);
      atomicAdd(gm + 3 * b.atom + x, t);
    }
  }
}

// One-electron part: each thread one ordered shell pair (I, J) of the CTA's molecule; the terms
// on the nuclei (nuclear attraction moving with the nucleus) and on the pair's centres collect
// in shared memory, then one atomic per component per molecule.
__global__ void __launch_bounds__(128)
k_grad_1e(const B2MolDev *__restrict__ mols, const B2Shell *__restrict__ shells,
          const double *__restrict__ atom_xyz, const int *__restrict__ atom_z, const double *__restrict__ btab,
          const double *__restrict__ D, const double *__restrict__ W, double *__restrict__ grad) {
  __shared__ double sZ[B2_MAXNAO], sR[3 * B2_MAXNAO], sG[3 * B2_MAXNAO];
  const B2MolDev md = mols[blockIdx.x];
  const int natm = md.natm, nbas = md.nbas, N = md.nao;
  for (int e = threadIdx.x; e < natm; e += blockDim.x) sZ[e] = (double)atom_z[md.atm_off + e];
  for (int e = threadIdx.x; e < 3 * natm; e += blockDim.x) {
    sR[e] = atom_xyz[3ll * md.atm_off + e];
    sG[e] = 0.0;
  }
  __syncthreads();
  const double *Dm = D + md.mat_off, *Wm = W + md.mat_off;
  for (int it = threadIdx.x; it < nbas * nbas; it += blockDim.x) {
    const int I = it / nbas, J = it - (it / nbas) * nbas;
    const B2Shell &a = shells[md.sh_off + I], &b = shells[md.sh_off + J];
    double g2[2][3];
    b2g_pair_grad_1e<double>(a, b, Dm, Wm, N, natm, sZ, sR, btab, g2,
                             [&](int c, int x, double v) { atomicAdd(&sG[3 * c + x], v); });
    for (int x = 0; x < 3; ++x) {
      atomicAdd(&sG[3 * a.atom + x], g2[0][x]);
      atomicAdd(&sG[3 * b.atom + x], g2[1][x]);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * natm; e += blockDim.x) atomicAdd(grad + 3ll * md.atm_off + e, sG[e]);
}

// Exchange-correlation part on 32 grid points of one molecule (tile t of molecule m, tile_off:
// per-molecule tile prefix).  With phi the AO values and u = D phi, U_k = D d_k phi:
//   rho = phi.u, grad rho = 2 (d phi).u, and moving atom A moves its orbitals, so
//   dE/dR_A,x = -2 sum_g w sum_{i on A} [vrho d_x phi_i u_i
//                                        + 2 vgamma sum_k g_k (d_x d_k phi_i u_i + d_x phi_i U_k,i)].
// Shared memory: D (N x N), phi and its gradient (4 x N x 32), u and U (4 x N x 32), the
// points' weighted vrho / vgamma and grad rho, and the molecule's atom sums.
__host__ __device__ inline long long b2g_xc_smem_doubles(int N, int natm) {
  return (long long)N * N + 8ll * N * B2G_TP + 5 * B2G_TP + 3ll * natm;
}

__global__ void __launch_bounds__(B2G_XC_THREADS)
k_grad_xc(const B2MolDev *__restrict__ mols, int nmol, const B2Shell *__restrict__ shells,
          const long long *__restrict__ grid_off, const long long *__restrict__ tile_off,
          const double *__restrict__ coords, const double *__restrict__ weights, const double *__restrict__ D,
          double *__restrict__ grad) {
  extern __shared__ double sm[];
  const long long bt = blockIdx.x;
  int lo = 0, hi = nmol - 1;                      // molecule: last m with tile_off[m] <= bt
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tile_off[mid] <= bt) lo = mid; else hi = mid - 1;
  }
  const int m = lo;
  const B2MolDev md = mols[m];
  const int N = md.nao, nbas = md.nbas, natm = md.natm;
  const long long p0 = grid_off[m] + (bt - tile_off[m]) * B2G_TP;
  const int np = (int)min((long long)B2G_TP, grid_off[m + 1] - p0);
  double *sD = sm;
  double *phi = sD + N * N;                       // [4][N][TP]
  double *u = phi + 4 * N * B2G_TP;               // [4][N][TP]
  double *vr = u + 4 * N * B2G_TP, *vg = vr + B2G_TP, *gr = vg + B2G_TP;   // gr [3][TP]
  double *sG = gr + 3 * B2G_TP;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int e = tid; e < N * N; e += blockDim.x) sD[e] = D[md.mat_off + e];
  for (int e = tid; e < 3 * natm; e += blockDim.x) sG[e] = 0.0;
  // AO values and gradients; item = shell * 32 + point, so a warp shares one shell
  for (int it = tid; it < nbas * B2G_TP; it += blockDim.x) {
    const int s = it / B2G_TP, p = it - s * B2G_TP;
    const B2Shell &S = shells[md.sh_off + s];
    double f[3] = {0, 0, 0}, df[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, hf[3][6];
    if (p < np) b2g_ao2<double>(S, coords + 3 * (p0 + p), f, df, hf);
    for (int c = 0; c < 2 * S.l + 1; ++c) {
      const int i = S.ao0 + c;
      phi[i * B2G_TP + p] = f[c];
      for (int x = 0; x < 3; ++x) phi[((1 + x) * N + i) * B2G_TP + p] = df[c][x];
    }
  }
  __syncthreads();
  for (int it = tid; it < N * B2G_TP; it += blockDim.x) {
    const int i = it / B2G_TP, p = it - i * B2G_TP;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int j = 0; j < N; ++j) {
      const double dij = sD[i * N + j];
      s0 += dij * phi[j * B2G_TP + p];
      s1 += dij * phi[(N + j) * B2G_TP + p];
      s2 += dij * phi[(2 * N + j) * B2G_TP + p];
      s3 += dij * phi[(3 * N + j) * B2G_TP + p];
    }
    u[i * B2G_TP + p] = s0;
    u[(N + i) * B2G_TP + p] = s1;
    u[(2 * N + i) * B2G_TP + p] = s2;
    u[(3 * N + i) * B2G_TP + p] = s3;
  }
  __syncthreads();
  if (tid < B2G_TP) {
    const int p = tid;
    double rho = 0, r1[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i) {
      const double ui = u[i * B2G_TP + p];
      rho += phi[i * B2G_TP + p] * ui;
      for (int x = 0; x < 3; ++x) r1[x] += phi[((1 + x) * N + i) * B2G_TP + p] * ui;
    }
    double a = 0, b = 0;
    if (p < np) {
      const B2XcPoint<double> o = b2_b3lyp_point<double>(rho, r1[0], r1[1], r1[2]);
      const double wt = weights[p0 + p];
      a = wt * o.vrho;
      b = wt * o.vgamma;
    }
    vr[p] = a;
    vg[p] = b;
    for (int x = 0; x < 3; ++x) gr[x * B2G_TP + p] = 2.0 * r1[x];
  }
  __syncthreads();
  const int hidx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  for (int it = tid; it < nbas * B2G_TP; it += blockDim.x) {    // warp-uniform shell
    const int s = it / B2G_TP, p = it - s * B2G_TP;
    const B2Shell &S = shells[md.sh_off + s];
    double acc[3] = {0, 0, 0};
    if (p < np) {
      double f[3], df[3][3], hf[3][6];
      b2g_ao2<double>(S, coords + 3 * (p0 + p), f, df, hf);
      const double a = vr[p], b2 = 2.0 * vg[p];
      const double g0 = gr[p], g1 = gr[B2G_TP + p], g2 = gr[2 * B2G_TP + p];
      for (int c = 0; c < 2 * S.l + 1; ++c) {
        const int i = S.ao0 + c;
        const double u0 = u[i * B2G_TP + p];
        const double uk[3] = {u[(N + i) * B2G_TP + p], u[(2 * N + i) * B2G_TP + p], u[(3 * N + i) * B2G_TP + p]};
        const double gk[3] = {g0, g1, g2};
        for (int x = 0; x < 3; ++x) {
          double q = 0;
          for (int k = 0; k < 3; ++k) q += gk[k] * (hf[c][hidx[x][k]] * u0 + df[c][x] * uk[k]);
          acc[x] += a * df[c][x] * u0 + b2 * q;
        }
      }
    }
    for (int x = 0; x < 3; ++x) {
      double v = acc[x];
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&sG[3 * S.atom + x], -2.0 * v);
    }
  }
  __syncthreads();
  for (int e = tid; e < 3 * natm; e += blockDim.x) atomicAdd(grad + 3ll * md.atm_off + e, sG[e]);
}

// nuclear repulsion: g_a = -sum_{b != a} Z_a Z_b (R_a - R_b) / |R_a - R_b|^3 (coincident atoms
// contribute nothing, as in the reference)
__global__ void __launch_bounds__(128)
k_grad_nuc(const B2MolDev *__restrict__ mols, const double *__restrict__ atom_xyz, const int *__restrict__ atom_z,
           double *__restrict__ grad) {
  const B2MolDev md = mols[blockIdx.x];
  const double *R = atom_xyz + 3ll * md.atm_off;
  const int *Z = atom_z + md.atm_off;
  for (int a = threadIdx.x; a < md.natm; a += blockDim.x) {
    double g[3] = {0, 0, 0};
    for (int b = 0; b < md.natm; ++b) {
      const double d[3] = {R[3 * a] - R[3 * b], R[3 * a + 1] - R[3 * b + 1], R[3 * a + 2] - R[3 * b + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (b == a || r2 == 0.0) continue;
      const double f = (double)Z[a] * Z[b] / (r2 * sqrt(r2));
      for (int x = 0; x < 3; ++x) g[x] -= f * d[x];
    }
    for (int x = 0; x < 3; ++x) atomicAdd(grad + 3ll * (md.atm_off + a) + x, g[x]);
  }
}

// Classes with L = l_I + l_J + l_K + l_L + 1 <= 3 (at most two p shells): the recursion arrays
// are small, so each lane takes one primitive quartet of the batch and runs both recursions in
// registers (every step and index fixed at compile time from the class's step table); after
// each batch the lanes' weighted [e0|f0] values are summed over the warp (a transpose through
// shared memory, 32 entries at a time) into the entry's owner lane.  Pair records, the horizontal recursion and the contraction are
// those of k_grad_2e.
template <typename S, int O>
__device__ __forceinline__ void b2g_vrr_lane_op(double *v, const double *X, const double *Y, double hb, double rb,
                                                const double *Xk, const double *Yk, double hk, double rk, double h3) {
  constexpr B2gOp op = S::op(O);
  if constexpr (op.mmax >= 0) {
    constexpr bool bra = O < S::NOB;
    const double x = bra ? X[op.dd] : Xk[op.dd], y = bra ? Y[op.dd] : Yk[op.dd];
    const double c = (double)op.c1 * (bra ? hb : hk), r = bra ? rb : rk, c3 = (double)op.c3 * h3;
#pragma unroll
    for (int m = 0; m <= op.mmax; ++m) {
      double t = x * v[op.s1 + m] + y * v[op.s1 + m + 1];
      if constexpr (op.s2 >= 0) t += c * (v[op.s2 + m] - r * v[op.s2 + m + 1]);
      if constexpr (op.s3 >= 0) t += c3 * v[op.s3 + m + 1];
      v[op.dst + m] = t;
    }
  }
}
template <typename S, int... O>
__device__ __forceinline__ void b2g_vrr_lane(double *v, const double *X, const double *Y, double hb, double rb,
                                             const double *Xk, const double *Yk, double hk, double rk, double h3,
                                             std::integer_sequence<int, O...>) {
  (b2g_vrr_lane_op<S, O>(v, X, Y, hb, rb, Xk, Yk, hk, rk, h3), ...);
}
__device__ __forceinline__ double b2g_warp_sum(double x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

template <int G>
__global__ void __launch_bounds__(128)
k_grad_2e_l(const B2EriTask *__restrict__ tasks, long long ntask, const B2MolDev *__restrict__ mols,
            const B2PairInfo *__restrict__ pinfo, const int *__restrict__ cls_list,
            const B2Shell *__restrict__ shells, const double *__restrict__ btab, const double *__restrict__ D,
            double hyb, double *__restrict__ grad) {
  using C2 = B2g2e<G>;
  constexpr int LA = C2::LA, LB = C2::LB, LC = C2::LC, LD = C2::LD, L = C2::L;
  static_assert(L <= 3, "per-lane form: small classes only");
  constexpr int na = 2 * LA + 1, nb = 2 * LB + 1, nc = 2 * LC + 1, nd = 2 * LD + 1, NCMP = na * nb * nc * nd;
  using SB = typename C2::SB;
  using SK = typename C2::SK;
  constexpr int NTOT = 3 * SB::NACC + 2 * SK::NACC, NCH = (NTOT + 31) / 32;
  constexpr int PER_WARP = NTOT + 2 * B2_MAXPRIM * B2_MAXPRIM * B2G_PP + 32 * 33;
  __shared__ double sbuf[4][PER_WARP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ti = (long long)blockIdx.x * 4 + w;
  if (ti >= ntask) return;                        // whole warp
  double *acc = sbuf[w], *bpr = acc + NTOT, *kpr = bpr + B2_MAXPRIM * B2_MAXPRIM * B2G_PP;
  double *red = kpr + B2_MAXPRIM * B2_MAXPRIM * B2G_PP;
  const B2EriTask tk = tasks[ti];
  const B2MolDev md = mols[tk.mol];
  const B2PairInfo bp = pinfo[md.sp_off + tk.IJ];
  const B2Shell &a = shells[md.sh_off + bp.I], &b = shells[md.sh_off + bp.J];
  const double *Dm = D + md.mat_off;
  const int N = md.nao;
  double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
  double AB[3], AB2 = 0;
  for (int x = 0; x < 3; ++x) { AB[x] = a.R[x] - b.R[x]; AB2 += AB[x] * AB[x]; }
  const int nbp = b2g_pairs_warp(a, b, AB2, bpr, lane);
  double *gm = grad + 3ll * md.atm_off;
  for (int kq = 0; kq < tk.count; ++kq) {
    const int KL = cls_list[md.sp_off + md.cls_start[tk.cls] + tk.start + kq];
    if (KL > tk.IJ) continue;                     // uniform over the warp
    const B2PairInfo kp = pinfo[md.sp_off + KL];
    const B2Shell &c = shells[md.sh_off + kp.I], &d = shells[md.sh_off + kp.J];
    double CD[3], CD2 = 0;
    for (int x = 0; x < 3; ++x) { CD[x] = c.R[x] - d.R[x]; CD2 += CD[x] * CD[x]; }
    const int nkp = b2g_pairs_warp(c, d, CD2, kpr, lane);
    double accu[NCH];                             // owner-lane sums: entry u = 32 k + lane
#pragma unroll
    for (int k = 0; k < NCH; ++k) accu[k] = 0.0;
    const int ncombo = nbp * nkp;
    for (int c0 = 0; c0 < ncombo; c0 += 32) {
      const int cb = c0 + lane;
      double vb[SB::NV], vk[SK::NV];
      double al2 = 0, be2 = 0, ga2 = 0;
      if (cb < ncombo) {
        const int ib = cb / nkp, ik = cb - (cb / nkp) * nkp;
        const double *B = bpr + ib * B2G_PP, *K = kpr + ik * B2G_PP;
        const double z = B[2], e = K[2], iz = B[10], ie = K[10];
        const double rs = rsqrt(z + e), inv = rs * rs;          // 1/sqrt(zeta+eta), 1/(zeta+eta)
        double PA[3], QC[3], WP[3], WQ[3], PQ2 = 0;
        for (int x = 0; x < 3; ++x) {
          const double P = B[3 + x], Q = K[3 + x];
          const double W = (z * P + e * Q) * inv;
          PA[x] = B[6 + x];
          QC[x] = K[6 + x];
          WP[x] = W - P;
          WQ[x] = W - Q;
          PQ2 += (P - Q) * (P - Q);
        }
        const double rho = z * e * inv;
        const double pref = 34.98683665524972 * iz * ie * rs * B[9] * K[9];   // 2 pi^(5/2) / (z e sqrt(z+e)) K K
        double F[L + 1];
        b2_boys<double, L, double>(rho * PQ2, btab, F);
        const double hb = 0.5 * iz, rb = e * inv, hk = 0.5 * ie, rk = z * inv, h3 = 0.5 * inv;
#pragma unroll
        for (int m = 0; m <= L; ++m) vb[m] = vk[m] = pref * F[m];
        b2g_vrr_lane<SB>(vb, PA, WP, hb, rb, QC, WQ, hk, rk, h3, std::make_integer_sequence<int, SB::NOP>{});
        b2g_vrr_lane<SK>(vk, PA, WP, hb, rb, QC, WQ, hk, rk, h3, std::make_integer_sequence<int, SK::NOP>{});
        al2 = 2.0 * B[0];
        be2 = 2.0 * B[1];
        ga2 = 2.0 * K[0];
      } else {
#pragma unroll
        for (int t = 0; t < SB::NV; ++t) vb[t] = 0.0;
#pragma unroll
        for (int t = 0; t < SK::NV; ++t) vk[t] = 0.0;
      }
      // weighted values of every entry u summed over the batch's quartets -> owner lane u % 32:
      // 32 entries at a time through a 32 x 33 shared-memory transpose (lane = row)
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
#pragma unroll
        for (int jj = 0; jj < 32; ++jj) {
          const int u = 32 * ch + jj;
          if (u < NTOT) {
            double x;
            if (u < 3 * SB::NACC) {
              const int q = u / SB::NACC, t = u - q * SB::NACC;
              x = vb[(t / SB::NF) * SB::SE + (t % SB::NF) * SB::SM] * (q == 0 ? 1.0 : (q == 1 ? al2 : be2));
            } else {
              const int q = (u - 3 * SB::NACC) / SK::NACC, t = u - 3 * SB::NACC - q * SK::NACC;
              x = vk[(t / SK::NF) * SK::SE + (t % SK::NF) * SK::SM] * (q == 0 ? 1.0 : ga2);
            }
            red[lane * 33 + jj] = x;
          }
        }
        __syncwarp();
        if (32 * ch + lane < NTOT) {
          double sum = 0.0;
#pragma unroll 8
          for (int r = 0; r < 32; ++r) sum += red[r * 33 + lane];
          accu[ch] += sum;
        }
        __syncwarp();
      }
    }
#pragma unroll
    for (int k = 0; k < NCH; ++k) {
      const int u = 32 * k + lane;
      if (u < NTOT) acc[u] = accu[k];
    }
    __syncwarp();
    const auto *aB = reinterpret_cast<const double (*)[SB::NE][SB::NF]>(acc);
    const auto *aK = reinterpret_cast<const double (*)[SK::NE][SK::NF]>(acc + 3 * SB::NACC);
    const double deg = (bp.I == bp.J ? 1.0 : 2.0) * (kp.I == kp.J ? 1.0 : 2.0) * (KL == tk.IJ ? 1.0 : 2.0);
    double gC[3] = {0, 0, 0}, g3[3] = {0, 0, 0};
    for (int cmp = lane; cmp < NCMP; cmp += 32) {
      const int id = cmp % nd, ic = (cmp / nd) % nc, ib = (cmp / (nd * nc)) % nb, ia = cmp / (nd * nc * nb);
      const int i = a.ao0 + ia, j = b.ao0 + ib, k = c.ao0 + ic, l = d.ao0 + id;
      const double gmv = deg * (0.5 * Dm[i * N + j] * Dm[k * N + l] -
                                0.125 * hyb * (Dm[i * N + l] * Dm[j * N + k] + Dm[i * N + k] * Dm[j * N + l]));
      if (gmv == 0.0) continue;
      int ea[3], eb[3], ec[3], ed[3];
      b2g_comp(LA, ia, ea); b2g_comp(LB, ib, eb); b2g_comp(LC, ic, ec); b2g_comp(LD, id, ed);
      for (int x = 0; x < 3; ++x) {
        int up[3], dn[3];
        for (int q = 0; q < 3; ++q) { up[q] = ea[q] + (q == x); dn[q] = ea[q] - (q == x); }
        double dA = b2g_hrr(aB, 1, up, eb, ec, ed, AB, CD);
        if (ea[x]) dA -= (double)ea[x] * b2g_hrr(aB, 0, dn, eb, ec, ed, AB, CD);
        for (int q = 0; q < 3; ++q) { up[q] = eb[q] + (q == x); dn[q] = eb[q] - (q == x); }
        double dB = b2g_hrr(aB, 2, ea, up, ec, ed, AB, CD);
        if (eb[x]) dB -= (double)eb[x] * b2g_hrr(aB, 0, ea, dn, ec, ed, AB, CD);
        for (int q = 0; q < 3; ++q) { up[q] = ec[q] + (q == x); dn[q] = ec[q] - (q == x); }
        double dC = b2g_hrr(aK, 1, ea, eb, up, ed, AB, CD);
        if (ec[x]) dC -= (double)ec[x] * b2g_hrr(aK, 0, ea, eb, dn, ed, AB, CD);
        gA[x] += gmv * dA;
        gB[x] += gmv * dB;
        gC[x] += gmv * dC;
        g3[x] -= gmv * (dA + dB + dC);
      }
    }
    for (int x = 0; x < 3; ++x) {
      const double u = b2g_warp_sum(gC[x]), t = b2g_warp_sum(g3[x]);
      if (lane == 0) {
        atomicAdd(gm + 3 * c.atom + x, u);
        atomicAdd(gm + 3 * d.atom + x, t);
      }
    }
    __syncwarp();                                 // acc and the pair records are rewritten next
  }
  for (int x = 0; x < 3; ++x) {
    const double u = b2g_warp_sum(gA[x]), t = b2g_warp_sum(gB[x]);
    if (lane == 0) {
      atomicAdd(gm + 3 * a.atom + x, u);
      atomicAdd(gm + 3 * b.atom + x, t);
    }
  }
}

template <int G>
static int b2g_launch_2e(const B2PlanDev &P, const double *D, double hyb, double *grad, cudaStream_t st) {
  const long long t0 = P.eri_goff32[G], n = P.eri_goff32[G + 1] - t0;
  if constexpr (B2g2e<G>::L <= 3) {
    if (n > 0) {
      k_grad_2e_l<G><<<(unsigned)((n + 3) / 4), 128, 0, st>>>(P.eri_tasks32 + t0, n, P.mols, P.pinfo, P.cls_list,
                                                             P.shells, P.boys, D, hyb, grad);
      b2_count_launches(1);
    }
  } else if (n > 0) {
    static bool attr[8] = {false};                 // per device: shared memory above 48 KB
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 8) return B2_ERR_CUDA;
    if (!attr[dev]) {
      if (cudaFuncSetAttribute(k_grad_2e<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B2g2e<G>::SMEM) !=
          cudaSuccess)
        return B2_ERR_CUDA;
      attr[dev] = true;
    }
    k_grad_2e<G><<<(unsigned)((n + 3) / 4), 128, B2g2e<G>::SMEM, st>>>(P.eri_tasks32 + t0, n, P.mols, P.pinfo,
                                                                       P.cls_list, P.shells, P.boys, D, hyb, grad);
    b2_count_launches(1);
  }
  if constexpr (G < 15) return b2g_launch_2e<G + 1>(P, D, hyb, grad, st);
  return B2_OK;
}

int b2_launch_grad(B2PlanDev &P, int parts, double hyb, const double *C, const double *mo_energy,
                   const double *coords, const double *weights, double *D, double *W, double *grad,
                   cudaStream_t st) {
  if (!D || !W || !grad || (parts & ~15)) return B2_ERR_ARG;
  if ((parts & 4) && (!coords || !weights || !P.g.grid_off)) return B2_ERR_ARG;
  const int nmol = P.h.nmol;
  B2_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(double) * 3 * std::max(1, P.h.n_atm), st));
  if (nmol == 0) return B2_OK;
  if (C) {
    if (!mo_energy) return B2_ERR_ARG;
    k_grad_dm<<<nmol, 256, 0, st>>>(P.mols, C, mo_energy, D, W);
    b2_count_launches(1);
  }
  if (parts & 1) {
    k_grad_1e<<<nmol, 128, 0, st>>>(P.mols, P.shells, P.atom_xyz, P.atom_z, P.boys, D, W, grad);
    b2_count_launches(1);
  }
  if (parts & 2) {
    int rc = b2_eri_tasks_ready(P, 32, st);        // canonical quartets grouped by class
    if (rc) return rc;
    rc = b2g_launch_2e<0>(P, D, hyb, grad, st);     // the 16 class combinations
    if (rc) return rc;
  }
  if (parts & 4) {
    std::vector<long long> toff(nmol + 1, 0);
    for (int m = 0; m < nmol; ++m) {
      const long long G = P.g.grid_off_h[m + 1] - P.g.grid_off_h[m];
      toff[m + 1] = toff[m] + (G + B2G_TP - 1) / B2G_TP;
    }
    if (toff[nmol] > 0) {
      if (toff[nmol] >= (1ll << 31)) return B2_ERR_SIZE;
      const size_t smem = sizeof(double) * (size_t)b2g_xc_smem_doubles(P.h.max_nao, P.h.max_natm);
      B2_CUDA_TRY(cudaFuncSetAttribute(k_grad_xc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      long long *dtoff = nullptr;
      B2_CUDA_TRY(b2_dmalloc_t(&dtoff, sizeof(long long) * (nmol + 1), st));
      // pageable source: the call returns once the data is staged, so toff may go out of scope
      cudaError_t e = cudaMemcpyAsync(dtoff, toff.data(), sizeof(long long) * (nmol + 1),
                                      cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) {
        k_grad_xc<<<(unsigned)toff[nmol], B2G_XC_THREADS, smem, st>>>(P.mols, nmol, P.shells, P.g.grid_off,
                                                                       dtoff, coords, weights, D, grad);
        b2_count_launches(1);
        e = cudaGetLastError();
      }
      b2_dfree(dtoff, st);
      if (e != cudaSuccess) return B2_ERR_CUDA;
    }
  }
  if (parts & 8) {
    k_grad_nuc<<<nmol, 128, 0, st>>>(P.mols, P.atom_xyz, P.atom_z, grad);
    b2_count_launches(1);
  }
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
