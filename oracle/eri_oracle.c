/* ERI oracle: FP64 CPU restatement of the reference's two-electron integrals.
 *
 * Test infrastructure only (tests, smoke() and the bench's CPU baseline use it as the
 * checker); the product never calls it.
 *
 * Computes the s8 unique-ERI list that the reference obtains from
 * ``mol.intor('int2e_sph', aosym='s8')`` (nanoDFT.py:285) or from its libcint port
 * ``int2e_sph`` (electron_repulsion/int2e_sph.cpp:6750, FP64 copy cpu_int2e_sph.cpp:7706),
 * for s and p shells (STO-3G).  The reference evaluates each shell quartet by Rys
 * quadrature (CINT2e_loop_nopt / CINTg0_2e, int2e_sph.cpp:2452-2719, 1785-1892); this
 * restatement evaluates the same integrals with the Head-Gordon-Pople scheme: Obara-Saika
 * vertical recursion per primitive quartet (Obara & Saika, J. Chem. Phys. 84, 3963
 * (1986)), contraction, then horizontal recursion (Head-Gordon & Pople, J. Chem. Phys.
 * 89, 5777 (1988)).  Inputs are the libcint atm/bas/env arrays (cpu_int2e_sph.cpp:47-88);
 * the angular factors 1/sqrt(4pi) (s) and sqrt(3/(4pi)) (p) that libcint applies in
 * CINTcommon_fac_sp are applied here too.  Output position of AO quartet (i,j,k,l):
 * ij(ij+1)/2+kl with ij = i(i+1)/2+j, i>=j, k>=l, ij>=kl (sparse_symmetric_ERI.py:13-16).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define ATM_SLOTS 6
#define BAS_SLOTS 8
#define PTR_COORD 1
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define PTR_EXP 5
#define PTR_COEFF 6

/* Cartesian components up to l = 2: index -> exponents */
static const int CART[10][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,1},
                                {2,0,0},{1,1,0},{1,0,1},{0,2,0},{0,1,1},{0,0,2}};
static int cart_index(int x, int y, int z) {
    int l = x + y + z;
    if (l == 0) return 0;
    if (l == 1) return x ? 1 : (y ? 2 : 3);
    if (x == 2) return 4; if (x == 1 && y == 1) return 5; if (x == 1) return 6;
    if (y == 2) return 7; if (y == 1) return 8; return 9;
}
static int ncart_upto(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }
static int cart_start(int l) { return l * (l + 1) * (l + 2) / 6; }

/* Boys function F_m(t), m = 0..mmax, double precision. */
void oracle_boys(int mmax, double t, double *f) {
    if (t < 40.0) {
        /* series for F_mmax: e^{-t} sum_k (2t)^k / prod_{i=0..k} (2mmax + 2i + 1) */
        double term = 1.0 / (2 * mmax + 1), sum = term;
        for (int k = 1; k < 400; k++) {
            term *= 2.0 * t / (2 * mmax + 2 * k + 1);
            sum += term;
            if (term < 1e-18 * sum) break;
        }
        double et = exp(-t);
        f[mmax] = et * sum;
        for (int m = mmax - 1; m >= 0; m--) f[m] = (2.0 * t * f[m + 1] + et) / (2 * m + 1);
    } else {
        double et = exp(-t);
        f[0] = 0.5 * sqrt(M_PI / t) * erf(sqrt(t));
        for (int m = 0; m < mmax; m++) f[m + 1] = ((2 * m + 1) * f[m] - et) / (2.0 * t);
    }
}

static const double FAC_SP[2] = {0.282094791773878143, 0.488602511902919921};

static void shell_quartet(const int *sh, const int *atm, const int *bas, const double *env,
                          double out[3][3][3][3]) {
    int l[4], np[4];
    const double *R[4], *ex[4], *cf[4];
    for (int q = 0; q < 4; q++) {
        const int *b = bas + BAS_SLOTS * sh[q];
        l[q] = b[ANG_OF]; np[q] = b[NPRIM_OF];
        R[q] = env + atm[ATM_SLOTS * b[ATOM_OF] + PTR_COORD];
        ex[q] = env + b[PTR_EXP]; cf[q] = env + b[PTR_COEFF];
    }
    const int lab = l[0] + l[1], lcd = l[2] + l[3], L = lab + lcd;
    const int ne = ncart_upto(lab), nf = ncart_upto(lcd);
    double AB[3], CD[3];
    for (int d = 0; d < 3; d++) { AB[d] = R[0][d] - R[1][d]; CD[d] = R[2][d] - R[3][d]; }
    double AB2 = AB[0]*AB[0] + AB[1]*AB[1] + AB[2]*AB[2];
    double CD2 = CD[0]*CD[0] + CD[1]*CD[1] + CD[2]*CD[2];
    double acc[10][10];                 /* contracted (e0|f0) */
    memset(acc, 0, sizeof(acc));
    for (int pa = 0; pa < np[0]; pa++) for (int pb = 0; pb < np[1]; pb++) {
        double a = ex[0][pa], b = ex[1][pb], z = a + b;
        double P[3], PA[3];
        for (int d = 0; d < 3; d++) { P[d] = (a * R[0][d] + b * R[1][d]) / z; PA[d] = P[d] - R[0][d]; }
        double Kab = exp(-a * b / z * AB2) * cf[0][pa] * cf[1][pb];
        for (int pc = 0; pc < np[2]; pc++) for (int pd = 0; pd < np[3]; pd++) {
            double c = ex[2][pc], dd = ex[3][pd], e = c + dd;
            double Q[3], QC[3], W[3], WP[3], WQ[3], PQ2 = 0;
            for (int d = 0; d < 3; d++) {
                Q[d] = (c * R[2][d] + dd * R[3][d]) / e; QC[d] = Q[d] - R[2][d];
                W[d] = (z * P[d] + e * Q[d]) / (z + e); WP[d] = W[d] - P[d]; WQ[d] = W[d] - Q[d];
                PQ2 += (P[d] - Q[d]) * (P[d] - Q[d]);
            }
            double rho = z * e / (z + e);
            double Kcd = exp(-c * dd / e * CD2) * cf[2][pc] * cf[3][pd];
            double pref = 2.0 * pow(M_PI, 2.5) / (z * e * sqrt(z + e)) * Kab * Kcd;
            double F[5];
            oracle_boys(L, rho * PQ2, F);
            /* v[e][f][m] = [e0|f0]^(m) */
            double v[10][10][5];
            for (int m = 0; m <= L; m++) v[0][0][m] = pref * F[m];
            /* bra VRR */
            for (int le = 1; le <= lab; le++)
                for (int ie = cart_start(le); ie < cart_start(le + 1); ie++) {
                    int ax = CART[ie][0], ay = CART[ie][1], az = CART[ie][2];
                    int d = ax ? 0 : (ay ? 1 : 2);
                    int e1[3] = {ax, ay, az}; e1[d]--;
                    int i1 = cart_index(e1[0], e1[1], e1[2]);
                    int i2 = -1;
                    if (e1[d] > 0) { int e2[3] = {e1[0], e1[1], e1[2]}; e2[d]--; i2 = cart_index(e2[0], e2[1], e2[2]); }
                    for (int m = 0; m <= L - le; m++) {
                        double t = PA[d] * v[i1][0][m] + WP[d] * v[i1][0][m + 1];
                        if (i2 >= 0) t += e1[d] / (2 * z) * (v[i2][0][m] - rho / z * v[i2][0][m + 1]);
                        v[ie][0][m] = t;
                    }
                }
            /* ket VRR */
            for (int lf = 1; lf <= lcd; lf++)
                for (int jf = cart_start(lf); jf < cart_start(lf + 1); jf++) {
                    int fx = CART[jf][0], fy = CART[jf][1], fz = CART[jf][2];
                    int d = fx ? 0 : (fy ? 1 : 2);
                    int f1[3] = {fx, fy, fz}; f1[d]--;
                    int j1 = cart_index(f1[0], f1[1], f1[2]);
                    int j2 = -1;
                    if (f1[d] > 0) { int f2[3] = {f1[0], f1[1], f1[2]}; f2[d]--; j2 = cart_index(f2[0], f2[1], f2[2]); }
                    for (int ie = 0; ie < ne; ie++) {
                        int ed = CART[ie][d];
                        int i3 = -1;
                        if (ed > 0) { int e3[3] = {CART[ie][0], CART[ie][1], CART[ie][2]}; e3[d]--; i3 = cart_index(e3[0], e3[1], e3[2]); }
                        int le = CART[ie][0] + CART[ie][1] + CART[ie][2];
                        for (int m = 0; m <= L - le - lf; m++) {
                            double t = QC[d] * v[ie][j1][m] + WQ[d] * v[ie][j1][m + 1];
                            if (j2 >= 0) t += f1[d] / (2 * e) * (v[ie][j2][m] - rho / e * v[ie][j2][m + 1]);
                            if (i3 >= 0) t += ed / (2 * (z + e)) * v[i3][j1][m + 1];
                            v[ie][jf][m] = t;
                        }
                    }
                }
            for (int ie = 0; ie < ne; ie++) for (int jf = 0; jf < nf; jf++) acc[ie][jf] += v[ie][jf][0];
        }
    }
    /* HRR: (a b| with b = p_j -> (a+1_j 0| + AB_j (a 0| ; same on the ket */
    int na = 2 * l[0] + 1, nb = 2 * l[1] + 1, nc = 2 * l[2] + 1, nd = 2 * l[3] + 1;
    double fac = FAC_SP[l[0]] * FAC_SP[l[1]] * FAC_SP[l[2]] * FAC_SP[l[3]];
    for (int ia = 0; ia < na; ia++) for (int ib = 0; ib < nb; ib++)
    for (int ic = 0; ic < nc; ic++) for (int id = 0; id < nd; id++) {
        int ea[3] = {0,0,0}, ec[3] = {0,0,0};
        if (l[0]) ea[ia]++;
        if (l[2]) ec[ic]++;
        /* bra terms: list of (cart index, weight) */
        int bi[2], nbt = 0; double bw[2];
        if (l[1] == 0) { bi[0] = cart_index(ea[0], ea[1], ea[2]); bw[0] = 1; nbt = 1; }
        else {
            int e2[3] = {ea[0], ea[1], ea[2]}; e2[ib]++;
            bi[0] = cart_index(e2[0], e2[1], e2[2]); bw[0] = 1;
            bi[1] = cart_index(ea[0], ea[1], ea[2]); bw[1] = AB[ib]; nbt = 2;
        }
        int ki[2], nkt = 0; double kw[2];
        if (l[3] == 0) { ki[0] = cart_index(ec[0], ec[1], ec[2]); kw[0] = 1; nkt = 1; }
        else {
            int f2[3] = {ec[0], ec[1], ec[2]}; f2[id]++;
            ki[0] = cart_index(f2[0], f2[1], f2[2]); kw[0] = 1;
            ki[1] = cart_index(ec[0], ec[1], ec[2]); kw[1] = CD[id]; nkt = 2;
        }
        double s = 0;
        for (int x = 0; x < nbt; x++) for (int y = 0; y < nkt; y++) s += bw[x] * kw[y] * acc[bi[x]][ki[y]];
        out[ia][ib][ic][id] = s * fac;
    }
}

static inline int64_t tri(int64_t a, int64_t b) { return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; }

/* All unique ERIs of one molecule into s8 (length n4 = n2(n2+1)/2, n2 = nao(nao+1)/2). */
int oracle_eri_s8(double *s8, const int *ao_loc, const int *atm, int natm, const int *bas,
                  int nbas, const double *env) {
    (void)natm;
    for (int I = 0; I < nbas; I++)
    for (int J = 0; J <= I; J++)
    for (int K = 0; K <= I; K++)
    for (int L = 0; L <= K; L++) {
        if (tri(K, L) > tri(I, J)) continue;
        int sh[4] = {I, J, K, L};
        double blk[3][3][3][3];
        shell_quartet(sh, atm, bas, env, blk);
        int di = ao_loc[I + 1] - ao_loc[I], dj = ao_loc[J + 1] - ao_loc[J];
        int dk = ao_loc[K + 1] - ao_loc[K], dl = ao_loc[L + 1] - ao_loc[L];
        for (int a = 0; a < di; a++) for (int b = 0; b < dj; b++)
        for (int c = 0; c < dk; c++) for (int d = 0; d < dl; d++) {
            int i = ao_loc[I] + a, j = ao_loc[J] + b, k = ao_loc[K] + c, l = ao_loc[L] + d;
            s8[tri(tri(i, j), tri(k, l))] = blk[a][b][c][d];
        }
    }
    return 0;
}
