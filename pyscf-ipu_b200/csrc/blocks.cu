// Block gather between two device arrays (b2_copy_blocks): used to carry the per-molecule
// state of molecules still iterating (s8 ERI lists, exchange lists) from one batch plan's
// layout into the next plan's when converged molecules retire and new ones take their slots.
#include <cstdint>
#include "device_plan.cuh"
#include "devmem.cuh"

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

// FP32 FMA peak of this GPU, measured (b2_fp32_peak): every SM full of threads, each running 8
// independent FMA chains; the result is stored only under a condition no value meets, so the
// work is kept.  Timed with CUDA events around one launch after a warm-up launch.
__global__ void __launch_bounds__(256)
k_fma_peak(int iters, float seed, float *__restrict__ sink) {
  float a[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) a[c] = seed + 0.001f * (float)(threadIdx.x + c);
  const float m = 0.9999f, b = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) a[c] = fmaf(a[c], m, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += a[c];
  if (s == -12345.0f) sink[blockIdx.x] = s;
}

int b2_measure_fp32_peak(double *tflops) {
  int dev = 0, nsm = 0;
  B2_CUDA_TRY(cudaGetDevice(&dev));
  B2_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  float *sink = nullptr;
  B2_CUDA_TRY(b2_dmalloc_t(&sink, sizeof(float) * 8 * nsm));
  cudaEvent_t e0, e1;
  B2_CUDA_TRY(cudaEventCreate(&e0));
  B2_CUDA_TRY(cudaEventCreate(&e1));
  const int iters = 4096, grid = 8 * nsm;
  k_fma_peak<<<grid, 256>>>(iters / 8, 1.0f, sink);           // warm-up
  B2_CUDA_TRY(cudaEventRecord(e0));
  k_fma_peak<<<grid, 256>>>(iters, 1.0f, sink);
  B2_CUDA_TRY(cudaEventRecord(e1));
  b2_count_launches(2);
  B2_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  B2_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b2_dfree(sink);
  const double flops = 2.0 * 16 * 8 * (double)iters * 256.0 * grid;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return B2_OK;
}
