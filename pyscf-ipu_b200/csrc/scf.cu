// Device-resident SCF step (sm_100a), FP64, one CTA per molecule.
//
// Follows the reference iteration (nanoDFT.py:40-102, dft.py:789-882):
//   H = H_core + (J - hyb/2 K) + V_xc
//   DIIS (nanoDFT.py:338-364): err = S D H - (S D H)^T stored in a ring of 9, B-matrix
//     row/column head+1 <- <err_k, err>, masked until filled, c = pinv(B)[0,:]
//     (pinv as jnp.linalg.pinv: singular values below 10*max(m,n)*eps*s_max dropped),
//     H <- sum_k c[k+1] H_k
//   C = L^T eigvec(L H L^T) with L = inv(cholesky(S)) (nanoDFT.py:69, 239)
//   D = 2 C_occ C_occ^T (nanoDFT.py:72)
// The eigensolver is a parallel cyclic Jacobi method (round-robin pair ordering) on the
// matrix held in shared memory; the reference uses jnp.linalg.eigh or TessellateIPU's
// Jacobi ipu_eigh (nanoDFT.py:370-393).
#include "device_plan.cuh"
#include "scf.cuh"

__device__ double b2_block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  for (int i = 0; i < nw; ++i) s += red[i];
  __syncthreads();
  return s;
}

__device__ double b2_block_max(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  for (int i = 0; i < nw; ++i) s = fmax(s, red[i]);
  __syncthreads();
  return s;
}

// C[N][N] = A * B (or A * B^T), all row-major in shared memory, ld = N
__device__ void b2_mm(const double *A, const double *B, double *C, int N, bool transB) {
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    const int r = e / N, c = e - (e / N) * N;
    double s = 0;
    if (transB)
      for (int k = 0; k < N; ++k) s += A[r * N + k] * B[c * N + k];
    else
      for (int k = 0; k < N; ++k) s += A[r * N + k] * B[k * N + c];
    C[e] = s;
  }
}

// rotation (c, s) zeroing A_pq (Golub & Van Loan, sym.schur2)
__device__ __host__ inline void b2_schur2(double app, double aqq, double apq, double &c, double &s) {
  if (apq == 0.0) { c = 1.0; s = 0.0; return; }
  const double tau = (aqq - app) / (2.0 * apq);
  double t;
  if (fabs(tau) > 1e150) t = 0.5 / tau;
  else t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
  c = 1.0 / sqrt(1.0 + t * t);
  s = t * c;
}

// parallel cyclic Jacobi on A (n x n, n even, leading dimension ld = n + 1) in shared memory;
// V (same layout) <- eigenvectors.  Rows/columns >= nreal are decoupled padding; the
// convergence norms use the nreal block only.  Stops when the off-diagonal Frobenius norm is
// below 1e-13 of the total (eigenvectors then accurate to ~1e-13), or after max_sweeps.
__device__ int b2_jacobi(double *A, double *V, int n, int nreal, double *rot, int *prs,
                         double *red, int max_sweeps) {
  const int ld = n + 1;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - (e / n) * n;
    V[r * ld + c] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int half = n / 2;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    double off = 0, tot = 0;
    for (int e = threadIdx.x; e < nreal * nreal; e += blockDim.x) {
      const int r = e / nreal, c = e - (e / nreal) * nreal;
      const double a = A[r * ld + c];
      tot += a * a;
      if (r != c) off += a * a;
    }
    off = b2_block_sum(off, red);
    tot = b2_block_sum(tot, red);
    if (off <= 1e-26 * tot || off < 1e-300) break;
    for (int r = 0; r < n - 1; ++r) {
      if (threadIdx.x < half) {
        // round-robin pairs: index 0 fixed, the others rotate by r (k - 1 + r < 2 (n - 1))
        const int k = threadIdx.x;
        int a = k - 1 + r, b = n - 2 - k + r;
        if (a >= n - 1) a -= n - 1;
        if (b >= n - 1) b -= n - 1;
        a = (k == 0) ? 0 : a + 1;
        b += 1;
        const int p = min(a, b), q = max(a, b);
        double c, s;
        const double apq = A[p * ld + q], app = A[p * ld + p], aqq = A[q * ld + q];
        if (fabs(apq) <= 1e-300 || apq * apq < 1e-34 * fabs(app * aqq)) {
          c = 1.0; s = 0.0;                         // already negligible
        } else {
          // sym.schur2 (Golub & Van Loan) with tau = d / b, d = aqq - app, b = 2 apq:
          // t = sign(tau) / (|tau| + sqrt(1 + tau^2)) = sign(tau) |b| / (|d| + sqrt(d^2 + b^2))
          // (one square root, one division; padding never gets here: its couplings are zero)
          const double d = aqq - app, bb = 2.0 * apq;
          const double sg = (d == 0.0 || ((d > 0.0) == (bb > 0.0))) ? 1.0 : -1.0;
          const double t = sg * fabs(bb) / (fabs(d) + sqrt(d * d + bb * bb));
          c = rsqrt(1.0 + t * t);
          s = t * c;
        }
        prs[2 * k] = p; prs[2 * k + 1] = q;
        rot[2 * k] = c; rot[2 * k + 1] = s;
      }
      __syncthreads();
      // one pass per round: block (k, l) of A (rows of pair k, columns of pair l) <- G_k A_kl G_l^T,
      // rows first then columns, exactly the arithmetic of a row pass followed by a column pass;
      // V's columns of pair l <- V G_l^T
      for (int e = threadIdx.x; e < half * half + n * half; e += blockDim.x) {
        if (e < half * half) {
          const int k = e / half, l = e - (e / half) * half;
          const int p = prs[2 * k], q = prs[2 * k + 1], pl = prs[2 * l], ql = prs[2 * l + 1];
          const double ck = rot[2 * k], sk = rot[2 * k + 1], cl = rot[2 * l], sl = rot[2 * l + 1];
          if (sk == 0.0 && sl == 0.0) continue;
          double a00 = A[p * ld + pl], a01 = A[p * ld + ql], a10 = A[q * ld + pl], a11 = A[q * ld + ql];
          if (sk != 0.0) {
            const double b00 = ck * a00 - sk * a10, b10 = sk * a00 + ck * a10;
            const double b01 = ck * a01 - sk * a11, b11 = sk * a01 + ck * a11;
            a00 = b00; a10 = b10; a01 = b01; a11 = b11;
          }
          if (sl != 0.0) {
            const double b00 = cl * a00 - sl * a01, b01 = sl * a00 + cl * a01;
            const double b10 = cl * a10 - sl * a11, b11 = sl * a10 + cl * a11;
            a00 = b00; a01 = b01; a10 = b10; a11 = b11;
          }
          A[p * ld + pl] = a00; A[p * ld + ql] = a01; A[q * ld + pl] = a10; A[q * ld + ql] = a11;
        } else {
          const int e2 = e - half * half, l = e2 / n, row = e2 - (e2 / n) * n;
          const double cl = rot[2 * l], sl = rot[2 * l + 1];
          if (sl == 0.0) continue;
          const int pl = prs[2 * l], ql = prs[2 * l + 1];
          const double vkp = V[row * ld + pl], vkq = V[row * ld + ql];
          V[row * ld + pl] = cl * vkp - sl * vkq;
          V[row * ld + ql] = sl * vkp + cl * vkq;
        }
      }
      __syncthreads();
    }
  }
  return sweep;
}

// cyclic Jacobi on the 10 x 10 DIIS matrix A (shared memory, row-major) run by one warp; V <- the
// eigenvectors.  Each rotation (p, q) is a row phase (rows p, q) then a column phase (columns
// p, q, and V); both are independent across k, so lane k < 10 does element k of each phase with
// the arithmetic of the one-thread loop: the result is identical to the serial sweep order.
// The convergence norm is summed serially by lane 0 (same order) and broadcast.
__device__ void b2_jacobi_small_warp(double *A, double *V) {
  constexpr int n = 10;
  const int k = threadIdx.x & 31;
  if (k < n)
    for (int j = 0; j < n; ++j) V[k * n + j] = (k == j) ? 1.0 : 0.0;
  __syncwarp();
  for (int sweep = 0; sweep < 50; ++sweep) {
    int done = 0;
    if (k == 0) {
      double off = 0, tot = 0;
      for (int i = 0; i < n * n; ++i) { tot += A[i] * A[i]; if (i / n != i % n) off += A[i] * A[i]; }
      done = (off <= 1e-28 * tot || off < 1e-300);
    }
    if (__shfl_sync(0xffffffffu, done, 0)) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p * n + q], app = A[p * n + p], aqq = A[q * n + q];
        if (fabs(apq) <= 1e-300 || fabs(apq) < 1e-18 * sqrt(fabs(app * aqq))) continue;
        double c, s;
        b2_schur2(app, aqq, apq, c, s);
        if (s == 0.0) continue;
        __syncwarp();
        if (k < n) {
          const double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        __syncwarp();
        if (k < n) {
          const double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
          const double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
        __syncwarp();
      }
  }
}

// ------------------------------------------------------------------ Fock + DIIS
// ring layout per molecule (offset mat_off * 9): errs[9][N*N], hams[9][N*N]; B: 100 doubles
__global__ void __launch_bounds__(256)
k_fock_diis(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
            const int *__restrict__ iter, double hyb, int use_diis, const double *__restrict__ Hcore,
            const double *__restrict__ S, const double *__restrict__ D, const double *__restrict__ J,
            const double *__restrict__ K, const double *__restrict__ Vxc, double *__restrict__ H,
            double *__restrict__ diffJK, double *__restrict__ ring_err, double *__restrict__ ring_h,
            double *__restrict__ Bmat, double *__restrict__ diis_err, const int *__restrict__ map) {
  const int m = map ? map[blockIdx.x] : blockIdx.x;
  if (active && !active[m]) return;
  extern __shared__ double sm[];
  __shared__ double red[32];
  __shared__ double sc[10];
  __shared__ double stmp[9];
  __shared__ double sA[100], sV[100];
  const B2MolDev md = mols[m];
  const int N = md.nao, NN = N * N;
  const long long mo = md.mat_off;
  double *sH = sm, *sS = sH + NN, *sD = sS + NN, *sT = sD + NN;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const double djk = J[mo + e] - 0.5 * hyb * K[mo + e];
    diffJK[mo + e] = djk;
    sH[e] = Hcore[mo + e] + djk + Vxc[mo + e];
    sS[e] = S[mo + e];
    sD[e] = D[mo + e];
  }
  __syncthreads();
  if (!use_diis) {
    for (int e = threadIdx.x; e < NN; e += blockDim.x) H[mo + e] = sH[e];
    return;
  }
  const int it = iter[m];
  const int nd = 9, head = it % nd;
  b2_mm(sS, sD, sT, N, false);          // S D
  __syncthreads();
  b2_mm(sT, sH, sS, N, false);          // S D H  (into sS)
  __syncthreads();
  double *er = ring_err + mo * nd, *hr = ring_h + mo * nd;
  double emax = 0;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    const double v = sS[a * N + b] - sS[b * N + a];
    sT[e] = v;
    emax = fmax(emax, fabs(v));
    er[(long long)head * NN + e] = v;
    hr[(long long)head * NN + e] = sH[e];
  }
  emax = b2_block_max(emax, red);
  __syncthreads();
  const int nfill = min(it + 1, nd);
  // the nine dot products <err_k, err_new> in one pass and one reduction (each thread's partial
  // sums, the warp shuffles and the sum over warps add in the same order as nine block sums)
  {
    __shared__ double red9[9][8];                   // 256 threads: 8 warps
    double s9[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) s9[k] = 0.0;
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {
      const double t = sT[e];
#pragma unroll
      for (int k = 0; k < 9; ++k)
        if (k < nfill) s9[k] += er[(long long)k * NN + e] * t;
    }
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      double v = s9[k];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) red9[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < nd) {
      double sum = 0;
      for (int i = 0; i < nw; ++i) sum += red9[threadIdx.x][i];
      stmp[threadIdx.x] = (threadIdx.x < nfill) ? sum : 0.0;
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    double *B = Bmat + (long long)m * 100;
    if (l < 10) {
      if (it == 0)
        for (int j = 0; j < 10; ++j) B[l * 10 + j] = (l == 0) == (j == 0) ? 0.0 : 1.0;
    }
    __syncwarp();
    if (l < nd) { B[(head + 1) * 10 + 1 + l] = stmp[l]; B[(1 + l) * 10 + head + 1] = stmp[l]; }
    __syncwarp();
    // masked copy: rows/columns of unfilled ring slots are zero
    for (int i = l; i < 100; i += 32) {
      const int r = i / 10, c = i - r * 10;
      const bool keep = (r == 0 || r - 1 < nfill) && (c == 0 || c - 1 < nfill);
      sA[i] = keep ? B[i] : 0.0;
    }
    __syncwarp();
    b2_jacobi_small_warp(sA, sV);
    __syncwarp();
    double smax = 0;
    for (int i = 0; i < 10; ++i) smax = fmax(smax, fabs(sA[i * 10 + i]));
    const double cut = 10.0 * 10.0 * 2.220446049250313e-16 * smax;
    if (l < 10) {
      double c = 0;
      for (int k = 0; k < 10; ++k) {
        const double lam = sA[k * 10 + k];
        if (fabs(lam) > cut) c += sV[0 * 10 + k] * sV[l * 10 + k] / lam;
      }
      sc[l] = c;
    }
    if (l == 0) diis_err[m] = emax;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    double s = 0;
    for (int k = 0; k < nfill; ++k) s += sc[k + 1] * hr[(long long)k * NN + e];
    H[mo + e] = s;
  }
}

// ------------------------------------------------------------------ eigensolve + density
// F' = L H L^T; with a previous eigenvector basis W (ws, per molecule) and iter > 0 the Jacobi
// sweeps run on W^T F' W, which is nearly diagonal once the SCF settles (2-3 sweeps instead of
// 6-8); the eigenvectors are W V'.  The result is the same eigen-decomposition up to the sign
// and order of eigenvectors, which the density does not depend on.
__global__ void __launch_bounds__(512)
k_eigh_density(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
               const int *__restrict__ iter, const double *__restrict__ H,
               const double *__restrict__ Linv, double *__restrict__ D, double *__restrict__ mo_energy,
               double *__restrict__ C, double *__restrict__ ws, int *__restrict__ sweeps,
               const int *__restrict__ map) {
  const int m = map ? map[blockIdx.x] : blockIdx.x;
  if (active && !active[m]) return;
  extern __shared__ double sm[];
  __shared__ double red[32];
  __shared__ double rot[B2_MAXNAO];
  __shared__ int prs[B2_MAXNAO];
  __shared__ int order[B2_MAXNAO];
  __shared__ double evals[B2_MAXNAO];
  const B2MolDev md = mols[m];
  const int N = md.nao, NN = N * N;
  const int n = (N + 1) & ~1;                     // even size for the round-robin ordering
  const int ld = n + 1;                            // odd leading dimension: no bank conflicts
  const long long mo = md.mat_off;
  const bool warm = ws && iter && iter[m] > 0;
  // shared memory holds A and V only; L and W are read from global memory (L1)
  double *sA = sm, *sV = sA + n * ld;
  const double *gL = Linv + mo, *gH = H + mo, *gW = ws ? ws + mo : nullptr;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {                         // L H -> sV
    const int r = e / N, c = e - (e / N) * N;
    double s = 0;
    for (int k = 0; k < N; ++k) s += gL[r * N + k] * gH[k * N + c];
    sV[r * ld + c] = s;
  }
  __syncthreads();
  // F' = (L H) L^T into sA (padded to n: decoupled padding sorts last); consecutive threads take
  // consecutive rows, so the L row is a broadcast and sV / sA are read and written conflict-free
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int c = e / n, r = e - (e / n) * n;
    double s = 0;
    if (r < N && c < N)
      for (int k = 0; k < N; ++k) s += sV[r * ld + k] * gL[c * N + k];
    else if (r == c)
      s = 1e30;
    sA[r * ld + c] = s;
  }
  __syncthreads();
  if (warm) {
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {                       // F' W -> sV
      const int r = e / N, c = e - (e / N) * N;
      double s = 0;
      for (int k = 0; k < N; ++k) s += sA[r * ld + k] * gW[k * N + c];
      sV[r * ld + c] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {                       // W^T (F' W) -> sA
      const int r = e / N, c = e - (e / N) * N;
      double s = 0;
      for (int k = 0; k < N; ++k) s += gW[k * N + r] * sV[k * ld + c];
      sA[r * ld + c] = s;
    }
    __syncthreads();
  }
  const int sw = b2_jacobi(sA, sV, n, N, rot, prs, red, 30);
  for (int i = threadIdx.x; i < n; i += blockDim.x) evals[i] = sA[i * ld + i];
  __syncthreads();
  // eigenvectors E in the orthogonal basis: W V' (warm) or V', into sA
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int r = e / N, c = e - (e / N) * N;
    double s;
    if (warm) {
      s = 0;
      for (int k = 0; k < N; ++k) s += gW[r * N + k] * sV[k * ld + c];
    } else {
      s = sV[r * ld + c];
    }
    sA[r * ld + c] = s;
  }
  __syncthreads();
  if (ws)
    for (int e = threadIdx.x; e < NN; e += blockDim.x) ws[mo + e] = sA[(e / N) * ld + e % N];
  // ascending order of eigenvalues: a total order (NaN sorts as +inf, ties by index), so the
  // ranks are a permutation of 0..n-1 whatever the values (every order[] slot is written)
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double li = evals[i] == evals[i] ? evals[i] : INFINITY;
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double lj = evals[j] == evals[j] ? evals[j] : INFINITY;
      rank += (lj < li) || (lj == li && j < i);
    }
    order[rank] = i;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < N; k += blockDim.x) mo_energy[(long long)m * B2_MAXNAO + k] = evals[order[k]];
  // C[:, k] = L^T E[:, order[k]]  (all N columns, into sV)
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int r = e / N, k = e - (e / N) * N;
    const int col = order[k];
    double s = 0;
    for (int a = 0; a < N; ++a) s += gL[a * N + r] * sA[a * ld + col];
    sV[r * ld + k] = s;
  }
  __syncthreads();
  const int nocc = md.nocc;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const int a = e / N, b = e - (e / N) * N;
    double s = 0;
    for (int k = 0; k < nocc; ++k) s += sV[a * ld + k] * sV[b * ld + k];
    D[mo + e] = 2.0 * s;
    if (C) C[mo + e] = sV[a * ld + b];
  }
  if (threadIdx.x == 0 && sweeps) sweeps[m] = sw;
}

// energies [E, E_core, E_J_K/2, E_xc, E_nuc] (nanoDFT.py:20-38)
__global__ void k_energy(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
                         const double *__restrict__ D, const double *__restrict__ Hcore,
                         const double *__restrict__ diffJK, const double *__restrict__ exc,
                         const double *__restrict__ enuc, double *__restrict__ out) {
  const int m = blockIdx.x;
  if (active && !active[m]) return;
  __shared__ double red[32];
  const B2MolDev md = mols[m];
  const int NN = md.nao * md.nao;
  double ec = 0, ej = 0;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const double d = D[md.mat_off + e];
    ec += d * Hcore[md.mat_off + e];
    ej += d * diffJK[md.mat_off + e];
  }
  ec = b2_block_sum(ec, red);
  ej = b2_block_sum(ej, red);
  if (threadIdx.x == 0) {
    double *o = out + (long long)m * 5;
    o[0] = ec + 0.5 * ej + exc[m] + enuc[m];
    o[1] = ec;
    o[2] = 0.5 * ej;
    o[3] = exc[m];
    o[4] = enuc[m];
  }
}

// end of one SCF iteration (nanoDFT.py:74-80): diff_JK = J - hyb/2 K of the new density
// (get_JK, nanoDFT.py:125-139), the five energy terms (nanoDFT.py:20-38) and the molecule's
// iteration counter advanced; inactive molecules are left untouched
__global__ void k_energy_jk(const B2MolDev *__restrict__ mols, const int *__restrict__ active,
                            const double *__restrict__ D, const double *__restrict__ Hcore,
                            const double *__restrict__ J, const double *__restrict__ K, double hyb,
                            const double *__restrict__ exc, const double *__restrict__ enuc,
                            double *__restrict__ diffJK, double *__restrict__ out, int *__restrict__ iter) {
  const int m = blockIdx.x;
  if (active && !active[m]) return;
  __shared__ double red[32];
  const B2MolDev md = mols[m];
  const int NN = md.nao * md.nao;
  double ec = 0, ej = 0;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) {
    const long long a = md.mat_off + e;
    const double d = D[a];
    const double djk = J[a] - 0.5 * hyb * K[a];
    diffJK[a] = djk;
    ec += d * Hcore[a];
    ej += d * djk;
  }
  ec = b2_block_sum(ec, red);
  ej = b2_block_sum(ej, red);
  if (threadIdx.x == 0) {
    double *o = out + (long long)m * 5;
    o[0] = ec + 0.5 * ej + exc[m] + enuc[m];
    o[1] = ec;
    o[2] = 0.5 * ej;
    o[3] = exc[m];
    o[4] = enuc[m];
    if (iter) iter[m] += 1;
  }
}

int b2_launch_energy_jk(const B2PlanDev &P, const int *active, const double *D, const double *Hcore,
                        const double *J, const double *K, double hyb, const double *exc,
                        const double *enuc, double *diffJK, double *out, int *iter, cudaStream_t st) {
  k_energy_jk<<<P.h.nmol, 256, 0, st>>>(P.mols, active, D, Hcore, J, K, hyb, exc, enuc, diffJK, out, iter);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

// L = inv(cholesky(S)) per molecule (FP64), one CTA per molecule (serial-ish, small N)
__global__ void k_chol_inv(const B2MolDev *__restrict__ mols, const double *__restrict__ S,
                           double *__restrict__ Linv, int *__restrict__ status) {
  const int m = blockIdx.x;
  extern __shared__ double sm[];
  const B2MolDev md = mols[m];
  const int N = md.nao, NN = N * N;
  double *sC = sm, *sI = sm + NN;
  for (int e = threadIdx.x; e < NN; e += blockDim.x) sC[e] = S[md.mat_off + e];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  // right-looking Cholesky: lower triangle of sC
  for (int k = 0; k < N; ++k) {
    if (threadIdx.x == 0) {
      const double d = sC[k * N + k];
      if (!(d > 0)) bad = 1;
      sC[k * N + k] = sqrt(fmax(d, 1e-300));
    }
    __syncthreads();
    const double dk = sC[k * N + k];
    for (int i = k + 1 + threadIdx.x; i < N; i += blockDim.x) sC[i * N + k] /= dk;
    __syncthreads();
    for (int e = threadIdx.x; e < (N - k - 1) * (N - k - 1); e += blockDim.x) {
      const int i = k + 1 + e / (N - k - 1), j = k + 1 + e % (N - k - 1);
      if (j <= i) sC[i * N + j] -= sC[i * N + k] * sC[j * N + k];
    }
    __syncthreads();
  }
  // inverse of the lower-triangular factor, column by column (forward substitution)
  for (int c = threadIdx.x; c < N; c += blockDim.x) {
    for (int i = 0; i < N; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) s -= sC[i * N + k] * sI[k * N + c];
      sI[i * N + c] = (i < c) ? 0.0 : s / sC[i * N + i];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NN; e += blockDim.x) Linv[md.mat_off + e] = sI[e];
  if (threadIdx.x == 0 && status) status[m] = bad ? B2_ERR_NOT_PD : B2_OK;
}

static size_t b2_fock_smem(int N) { return sizeof(double) * 4 * N * N; }
static size_t b2_eigh_smem(int N) { int n = (N + 1) & ~1; return sizeof(double) * 2 * n * (n + 1); }

// One launch per orbital bucket (nao <= 16, 32, 48, 64, more) with shared memory sized for that
// bucket, so small molecules run several CTAs per SM.  The bucket launches go to the plan's
// bucket streams, forked from and joined back to the caller's stream with events, so they run
// concurrently (a serial sequence of launches would leave the GPU idle at each launch's tail).
template <typename F>
static int b2_per_bucket(const B2PlanDev &P, cudaStream_t st, F launch) {
  const bool sub = P.sub.n > 0;
  const std::vector<int> &off = sub ? P.sub.bkt_off_h : P.bkt_off_h;
  const int *map = sub ? P.sub.bkt_map : P.bkt_map;
  B2_CUDA_TRY(cudaEventRecord(P.bkt_ev[B2_NBKT], st));
  for (int b = B2_NBKT - 1; b >= 0; --b) {          // largest molecules first
    const int n = off[b + 1] - off[b];
    if (n <= 0) continue;
    const int N = std::min(P.h.max_nao, 16 * (b + 1));
    B2_CUDA_TRY(cudaStreamWaitEvent(P.bkt_stream[b], P.bkt_ev[B2_NBKT], 0));
    launch(N, n, map + off[b], P.bkt_stream[b]);
    b2_count_launches(1);
    B2_CUDA_TRY(cudaGetLastError());
    B2_CUDA_TRY(cudaEventRecord(P.bkt_ev[b], P.bkt_stream[b]));
    B2_CUDA_TRY(cudaStreamWaitEvent(st, P.bkt_ev[b], 0));
  }
  return B2_OK;
}

int b2_launch_fock_diis(const B2PlanDev &P, const int *active, const int *iter, double hyb,
                        int use_diis, const double *Hcore, const double *S, const double *D,
                        const double *J, const double *K, const double *Vxc, double *H,
                        double *diffJK, double *ring_err, double *ring_h, double *Bmat,
                        double *diis_err, cudaStream_t st) {
  B2_CUDA_TRY(cudaFuncSetAttribute(k_fock_diis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)b2_fock_smem(P.h.max_nao)));
  return b2_per_bucket(P, st, [&](int N, int n, const int *map, cudaStream_t s) {
    k_fock_diis<<<n, 256, b2_fock_smem(N), s>>>(P.mols, active, iter, hyb, use_diis, Hcore, S, D, J, K,
                                                Vxc, H, diffJK, ring_err, ring_h, Bmat, diis_err, map);
  });
}

int b2_launch_eigh_density(const B2PlanDev &P, const int *active, const int *iter, const double *H,
                           const double *Linv, double *D, double *mo_energy, double *C, double *ws,
                           int *sweeps, cudaStream_t st) {
  B2_CUDA_TRY(cudaFuncSetAttribute(k_eigh_density, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)b2_eigh_smem(P.h.max_nao)));
  return b2_per_bucket(P, st, [&](int N, int n, const int *map, cudaStream_t s) {
    k_eigh_density<<<n, N > 32 ? 512 : 256, b2_eigh_smem(N), s>>>(P.mols, active, iter, H, Linv, D, mo_energy, C, ws,
                                                   sweeps, map);
  });
}

int b2_launch_energy(const B2PlanDev &P, const int *active, const double *D, const double *Hcore,
                     const double *diffJK, const double *exc, const double *enuc, double *out,
                     cudaStream_t st) {
  k_energy<<<P.h.nmol, 256, 0, st>>>(P.mols, active, D, Hcore, diffJK, exc, enuc, out);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}

int b2_launch_chol_inv(const B2PlanDev &P, const double *S, double *Linv, int *status,
                       cudaStream_t st) {
  size_t sm = sizeof(double) * 2 * P.h.max_nao * P.h.max_nao;
  B2_CUDA_TRY(cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_chol_inv<<<P.h.nmol, 128, sm, st>>>(P.mols, S, Linv, status);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
