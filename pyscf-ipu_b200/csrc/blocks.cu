// Block gather between two device arrays (b2_copy_blocks): used to carry the per-molecule
// state of molecules still iterating (s8 ERI lists, exchange lists) from one batch plan's
// layout into the next plan's when converged molecules retire and new ones take their slots.
#include <cstdint>
#include "device_plan.cuh"

// one CTA per block: 16-byte vectors over the 16-byte-aligned middle, single bytes at the ends
__global__ void __launch_bounds__(256)
k_copy_blocks(const unsigned char *__restrict__ src, unsigned char *__restrict__ dst,
              const long long *__restrict__ src_off, const long long *__restrict__ dst_off,
              const long long *__restrict__ len) {
  const long long so = src_off[blockIdx.x], doff = dst_off[blockIdx.x], n = len[blockIdx.x];
  const unsigned char *s = src + so;
  unsigned char *d = dst + doff;
  // vector path only when source and destination share their offset modulo 16
  const long long head = ((16 - (reinterpret_cast<uintptr_t>(s) & 15)) & 15);
  if (((reinterpret_cast<uintptr_t>(s) ^ reinterpret_cast<uintptr_t>(d)) & 15) == 0 && n > head + 16) {
    for (long long i = threadIdx.x; i < head; i += blockDim.x) d[i] = s[i];
    const long long nv = (n - head) >> 4;
    const uint4 *sv = reinterpret_cast<const uint4 *>(s + head);
    uint4 *dv = reinterpret_cast<uint4 *>(d + head);
    for (long long i = threadIdx.x; i < nv; i += blockDim.x) dv[i] = sv[i];
    for (long long i = head + (nv << 4) + threadIdx.x; i < n; i += blockDim.x) d[i] = s[i];
  } else {
    for (long long i = threadIdx.x; i < n; i += blockDim.x) d[i] = s[i];
  }
}

int b2_launch_copy_blocks(int n, const void *src, void *dst, const long long *src_off,
                          const long long *dst_off, const long long *len, cudaStream_t st) {
  if (n <= 0) return B2_OK;
  k_copy_blocks<<<n, 256, 0, st>>>((const unsigned char *)src, (unsigned char *)dst, src_off, dst_off, len);
  b2_count_launches(1);
  B2_CUDA_TRY(cudaGetLastError());
  return B2_OK;
}
