// Shared definitions for the b200dft CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#define B2_HD __host__ __device__ __forceinline__

// status codes returned across the C ABI
enum {
  B2_OK = 0,
  B2_ERR_ARG = -1,
  B2_ERR_CUDA = -2,
  B2_ERR_UNSUPPORTED = -3,
  B2_ERR_SIZE = -4,
  B2_ERR_NOT_PD = -5,
  B2_ERR_TIMEOUT = -6,
};

// libcint slots (pyscf_ipu/electron_repulsion/cpu_int2e_sph.cpp:47-88)
#define B2_ATM_SLOTS 6
#define B2_BAS_SLOTS 8
#define B2_PTR_COORD 1
#define B2_ATOM_OF 0
#define B2_ANG_OF 1
#define B2_NPRIM_OF 2
#define B2_NCTR_OF 3
#define B2_PTR_EXP 5
#define B2_PTR_COEFF 6

#define B2_MAXPRIM 3          // STO-3G: 3 primitives per shell
#define B2_MAXPP 9            // primitive pairs per shell pair
#define B2_MAXNAO 72          // nao <= 70 (north star cap), padded
#define B2_MAXL 1             // s and p shells

// angular factors libcint applies on top of the radial normalisation (CINTcommon_fac_sp)
#define B2_FAC_S 0.282094791773878143
#define B2_FAC_P 0.488602511902919921

struct B2Shell {               // one contracted shell of one molecule
  double R[3];
  double exp[B2_MAXPRIM];
  double coef[B2_MAXPRIM];     // libcint coefficient * angular factor
  int l, ao0, nprim, atom;
};

// primitive-pair data of a shell pair (bra or ket), precision T; 16-byte aligned (48 / 96
// bytes) so that kernels load it with 128-bit vector loads
template <typename T>
struct __align__(16) B2PairPrim {
  T zeta, Px, Py, Pz, K, PAx, PAy, PAz, PBx, PBy, PBz, h2z;   // h2z = 1 / (2 zeta)
};

struct B2PairInfo {            // per shell pair
  int I, J, lI, lJ, ao0I, ao0J, nprim, pad;
};

B2_HD int64_t b2_tri(int64_t a) { return a * (a + 1) / 2; }

// inverse of tri: largest i with i(i+1)/2 <= p
B2_HD int64_t b2_untri(int64_t p) {
  int64_t i = (int64_t)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
  while (b2_tri(i + 1) <= p) ++i;
  while (b2_tri(i) > p) --i;
  return i;
}

#define B2_CUDA_TRY(x)                                         \
  do {                                                         \
    cudaError_t _e = (x);                                      \
    if (_e != cudaSuccess) return B2_ERR_CUDA;                 \
  } while (0)
