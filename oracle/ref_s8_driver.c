/* Test infrastructure (oracle): drive the reference's own FP64 ERI routine
 * ``int2e_sph`` (pyscf_ipu/electron_repulsion/cpu_int2e_sph.cpp:7706, built by
 * oracle/build_ref.py into oracle/_ref/libref_int2e.so) over every canonical shell
 * quartet of a molecule and scatter the blocks into the s8 unique-ERI list that
 * ``mol.intor('int2e_sph', aosym='s8')`` returns (nanoDFT.py:285).
 *
 * Block layout: int2e_sph writes component (ci,cj,ck,cl) at
 * out[ci + di*(cj + dj*(ck + dk*cl))] (consumed this way at int2e_sph.cpp:7649).
 * s8 position of AO quartet (i,j,k,l): ij = i(i+1)/2+j (i>=j), kl likewise,
 * pos = ij(ij+1)/2 + kl (ij>=kl) (decoded at sparse_symmetric_ERI.py:13-16).
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

extern int int2e_sph(double *out, int n_out, int *dims, int *shls, int *atm, int natm,
                     int *bas, int nbas, double *env, int n_env);

static inline int64_t tri(int64_t a, int64_t b) { return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; }

int ref_eri_s8(double *s8, const int *ao_loc, int *atm, int natm, int *bas, int nbas,
               double *env, int n_env) {
    double buf[4096];
    int64_t nq = 0;
    for (int I = 0; I < nbas; I++)
    for (int J = 0; J <= I; J++)
    for (int K = 0; K <= I; K++)
    for (int L = 0; L <= K; L++) {
        if (tri(K, L) > tri(I, J)) continue;
        int shls[4] = {I, J, K, L};
        memset(buf, 0, sizeof(buf));
        int di = ao_loc[I + 1] - ao_loc[I], dj = ao_loc[J + 1] - ao_loc[J];
        int dk = ao_loc[K + 1] - ao_loc[K], dl = ao_loc[L + 1] - ao_loc[L];
        int_fast8_t nonzero = (int_fast8_t)int2e_sph(buf, 4096, NULL, shls, atm, natm, bas, nbas, env, n_env);
        nq++;
        for (int cl = 0; cl < dl; cl++)
        for (int ck = 0; ck < dk; ck++)
        for (int cj = 0; cj < dj; cj++)
        for (int ci = 0; ci < di; ci++) {
            int i = ao_loc[I] + ci, j = ao_loc[J] + cj, k = ao_loc[K] + ck, l = ao_loc[L] + cl;
            double v = nonzero ? buf[ci + di * (cj + dj * (ck + dk * cl))] : 0.0;
            s8[tri(tri(i, j), tri(k, l))] = v;
        }
    }
    return (int)nq;
}

/* One shell quartet, raw block (for known-answer checks). */
int ref_int2e_block(double *out, int n_out, int *shls, int *atm, int natm, int *bas, int nbas,
                    double *env, int n_env) {
    return int2e_sph(out, n_out, NULL, shls, atm, natm, bas, nbas, env, n_env);
}
