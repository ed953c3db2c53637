// host_staging.h -- large copies between pageable host memory and the device
// through two pinned 64 MiB chunks: the DMA of one chunk overlaps the copy of
// the other between pinned and pageable memory, which runs on all OpenMP
// threads (so first touch of fresh pageable pages is parallel too).  Used by
// the mesh set-up paths, whose arrays reach several GB.
#ifndef CGX_HOST_STAGING_H
#define CGX_HOST_STAGING_H

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>

namespace cgx_staging {

inline void par_memcpy(void* dst, const void* src, size_t bytes) {
  const size_t blk = size_t(1) << 20;
  const long long nb = (long long)((bytes + blk - 1) / blk);
#pragma omp parallel for schedule(static)
  for (long long b = 0; b < nb; ++b) {
    const size_t off = size_t(b) * blk;
    std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, std::min(blk, bytes - off));
  }
}

class Staging {
 public:
  static constexpr size_t kChunk = size_t(64) << 20;

  explicit Staging(cudaStream_t s) : s_(s) {}
  Staging(const Staging&) = delete;
  Staging& operator=(const Staging&) = delete;

  // pinned buffers and events; must succeed before put/get
  cudaError_t init() {
    for (int i = 0; i < 2; ++i) {
      cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&pin_[i]), kChunk);
      if (e != cudaSuccess) return e;
      e = cudaEventCreateWithFlags(&done_[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  ~Staging() {
    cudaStreamSynchronize(s_);  // no DMA may still target the buffers
    for (int i = 0; i < 2; ++i) {
      if (pin_[i]) cudaFreeHost(pin_[i]);
      if (done_[i]) cudaEventDestroy(done_[i]);
    }
  }

  // host -> device, asynchronous on the stream (src may be reused on return)
  cudaError_t put(void* dst, const void* src, size_t bytes) {
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    for (size_t c = 0; c < nch; ++c) {
      const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
      cudaError_t e = cudaEventSynchronize(done_[c & 1]);  // the buffer's previous DMA
      if (e != cudaSuccess) return e;
      par_memcpy(pin_[c & 1], static_cast<const char*>(src) + off, len);
      e = cudaMemcpyAsync(static_cast<char*>(dst) + off, pin_[c & 1], len, cudaMemcpyHostToDevice, s_);
      if (e != cudaSuccess) return e;
      e = cudaEventRecord(done_[c & 1], s_);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  // device -> host, complete on return; on `st` instead of the object's
  // stream when given (the copies then follow st's earlier work)
  cudaError_t get(void* dst, const void* src, size_t bytes, cudaStream_t st = nullptr) {
    cudaStream_t q = st ? st : s_;
    const size_t nch = (bytes + kChunk - 1) / kChunk;
    for (size_t c = 0; c < nch; ++c) {
      const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
      cudaError_t e = cudaMemcpyAsync(pin_[c & 1], static_cast<const char*>(src) + off, len,
                                      cudaMemcpyDeviceToHost, q);
      if (e != cudaSuccess) return e;
      e = cudaEventRecord(done_[c & 1], q);
      if (e != cudaSuccess) return e;
      if (c > 0 && (e = drain(static_cast<char*>(dst), c - 1, bytes)) != cudaSuccess) return e;
    }
    return nch > 0 ? drain(static_cast<char*>(dst), nch - 1, bytes) : cudaSuccess;
  }

 private:
  cudaError_t drain(char* dst, size_t c, size_t bytes) {
    const size_t off = c * kChunk, len = std::min(kChunk, bytes - off);
    const cudaError_t e = cudaEventSynchronize(done_[c & 1]);
    if (e != cudaSuccess) return e;
    par_memcpy(dst + off, pin_[c & 1], len);
    return cudaSuccess;
  }

  cudaStream_t s_;
  char* pin_[2] = {nullptr, nullptr};
  cudaEvent_t done_[2] = {nullptr, nullptr};
};

}  // namespace cgx_staging

#endif
