// context.hpp — library context, device buffers and error plumbing.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "counters.hpp"
#include "ntt.cuh"
#include "stark_gpu.h"

struct sg_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // created on first use: host-to-device copies overlapped with compute
  // powers of the last LDE coset shift (two 2^14-entry tables), kept on the device
  uint64_t shift_key = 0;
  uint64_t* shift_tab = nullptr;
  std::vector<uint64_t> shift_host;
  sg::NttTables tw;
  bool owns_tables = true;  // worker contexts of a server borrow the parent's tables
  int wide_merge = SG_WIDE_MERGE_AUTO;  // SG_OPT_WIDE_MERGE
  int stir_group = 1;                   // SG_OPT_STIR_GROUP (servers created from this context)
  // Server workers only (null elsewhere): a highest-priority stream for the STIR
  // phase of a proof and the two events that order it after and before `stream`.
  cudaStream_t stir_stream = nullptr;
  cudaEvent_t stir_in = nullptr, stir_out = nullptr;
  // grow-only pinned host staging for witnesses copied to the device (pinned_host)
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  std::string err;
};

namespace sg {

struct SgError {
  int code;
  std::string msg;
};

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw SgError{SG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}
inline void require(bool ok, const std::string& msg) {
  if (!ok) throw SgError{SG_EINVAL, msg};
}

// Stream-ordered device buffer from the device's default memory pool.
struct DBuf {
  uint64_t* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DBuf() = default;
  DBuf(size_t elems, cudaStream_t st) { alloc(elems, st); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; }
  DBuf& operator=(DBuf&& o) noexcept {
    release();
    p = o.p;
    n = o.n;
    s = o.s;
    o.p = nullptr;
    return *this;
  }
  void alloc(size_t elems, cudaStream_t st) {
    release();
    s = st;
    n = elems;
    if (elems == 0) return;
    cudaError_t e = cudaMallocAsync((void**)&p, elems * sizeof(uint64_t), st);
    if (e != cudaSuccess) {
      p = nullptr;
      throw SgError{SG_ENOMEM, std::string("device allocation of ") + std::to_string(elems * 8) +
                                   " bytes failed: " + cudaGetErrorString(e)};
    }
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
  }
  ~DBuf() { release(); }
};

bool is_device_ptr(const void* p);

// The context's pinned host staging buffer, grown to at least `bytes`. Earlier
// contents are not kept; the caller synchronises its stream before the next use.
void* pinned_host(sg_ctx* c, size_t bytes);
// Give the context's staging buffer back to the process-wide pool.
void pinned_release(sg_ctx* c);

// sg_pool_reserve: grow the device's default pool to `bytes` (best effort).
void pool_reserve(int device, uint64_t bytes, cudaStream_t s);

}  // namespace sg
