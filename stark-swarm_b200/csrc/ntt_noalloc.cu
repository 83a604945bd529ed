// ntt_noalloc.cu — sg_ntt_noalloc: the batched NTT without any device allocation.
//
// Some callers cannot let this library allocate device memory: a serving
// process that has already divided all of HBM between proof jobs, a host
// framework (for example a Rust worker reaching this code over FFI) whose own
// allocator owns every device buffer, or a latency-critical loop where
// cudaMalloc's implicit device-wide synchronisation is not acceptable. For
// them this entry point runs the same two-pass NTT kernels as sg_ntt, but the
// transpose buffer between the passes and the twiddle tables live in
// file-scope static device arrays of fixed size, so nothing is allocated per
// call. The arrays are created when the library is loaded and every GPU that
// loads it keeps them (kNoAllocScratchElems * 8 bytes + 576 KiB) until exit.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "gl.cuh"
#include "ntt.cuh"
#include "stark_gpu.h"

namespace {

// 2^20 elements = 8 MiB: enough for n_cols * 2^log_n <= 2^20 on transforms
// longer than 2^12 (shorter transforms need no scratch at all).
constexpr size_t kNoAllocScratchElems = size_t(1) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint64_t g_noalloc_scratch[kNoAllocScratchElems];
static __device__ __align__(256) uint64_t g_noalloc_twiddles[2 * sg::kTwDirElems];

struct DeviceSlot {
  bool ready = false;
  uint64_t* scratch = nullptr;   // device address of g_noalloc_scratch on this device
  uint64_t* twiddles = nullptr;  // device address of g_noalloc_twiddles on this device
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_mu;
uint64_t g_host_twiddles[2 * sg::kTwDirElems];  // layout of sg::ntt_tables_host
bool g_host_twiddles_ready = false;

// Once per device, with that device current: resolve the device addresses of
// the static arrays (host code may not use the symbols' names as pointers) and
// fill the twiddle table. Runs inside the first sg_ntt_noalloc call on a device.
int setup_device(int dev) {
  std::lock_guard<std::mutex> g(g_mu);
  DeviceSlot& s = g_slots[dev];
  if (s.ready) return SG_OK;
  if (!g_host_twiddles_ready) {
    sg::ntt_tables_host(g_host_twiddles);
    g_host_twiddles_ready = true;
  }
  uint64_t* scratch = nullptr;
  uint64_t* tw = nullptr;
  if (cudaGetSymbolAddress((void**)&scratch, g_noalloc_scratch) != cudaSuccess) return SG_ECUDA;
  if (cudaGetSymbolAddress((void**)&tw, g_noalloc_twiddles) != cudaSuccess) return SG_ECUDA;
  if (cudaMemcpy(tw, g_host_twiddles, sizeof g_host_twiddles, cudaMemcpyHostToDevice) != cudaSuccess)
    return SG_ECUDA;
  s.scratch = scratch;
  s.twiddles = tw;
  s.ready = true;
  return SG_OK;
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int sg_ntt_noalloc(const uint64_t* d_in, uint64_t* d_out, size_t n_cols, size_t log_n, int inverse,
                              void* cuda_stream) {
  if (!d_in || !d_out || n_cols == 0 || n_cols >= (size_t(1) << 31) || log_n > (size_t)sg::kMaxLogN)
    return SG_EINVAL;
  const size_t n = size_t(1) << log_n;
  if (sg::ntt_scratch_elems(n_cols, (int)log_n) > kNoAllocScratchElems) return SG_ELIMIT;
  if (!on_device(d_in) || !on_device(d_out)) return SG_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SG_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return SG_EINVAL;
  const int rc = setup_device(dev);
  if (rc != SG_OK) return rc;
  const DeviceSlot& s = g_slots[dev];
  const sg::NttTables t = sg::ntt_tables_view(s.twiddles);
  // Pass 1 writes every scratch element that pass 2 reads, so the scratch left
  // by an earlier call needs no clearing.
  const cudaError_t e = sg::ntt_batch(t, d_in, d_out, (uint32_t)n_cols, n, n, (int)log_n, inverse != 0, n,
                                      log_n > 12 ? s.scratch : nullptr, (cudaStream_t)cuda_stream);
  return e == cudaSuccess ? SG_OK : SG_ECUDA;
}
