// Device memory of plans and grid tables.
//
// Every table a plan owns comes from one stream-ordered memory pool per device whose freed
// blocks stay mapped (release threshold: unlimited).  Consecutive batches' plans then reuse the
// same memory: no cudaFree (which synchronizes the device and unmaps pages) between batches.
// The pool does not add internal dependencies between streams: a block freed on one stream is
// handed to an allocation on another only once its free has completed, so a plan built on a
// worker thread never waits for the batch running on the GPU.  b2_release_cached_memory returns
// the unused blocks to the driver.
#pragma once
#include <cuda_runtime.h>

// allocate `bytes` in stream order on `st` (nullptr: the legacy default stream)
cudaError_t b2_dmalloc(void **p, size_t bytes, cudaStream_t st = nullptr);
// free in stream order on `st` (nullptr: the legacy default stream, i.e. after all work queued
// on blocking streams); nullptr pointers are ignored
void b2_dfree(void *p, cudaStream_t st = nullptr);

template <typename T>
inline cudaError_t b2_dmalloc_t(T **p, size_t bytes, cudaStream_t st = nullptr) {
  return b2_dmalloc(reinterpret_cast<void **>(p), bytes, st);
}
