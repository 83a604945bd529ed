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
#include <cuda.h>  // CUcontext and CUresult types; no libcuda link
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
  unsigned long long ctx_id = 0;  // context the arrays were set up in (0: unknown)
  uint64_t* scratch = nullptr;    // device address of g_noalloc_scratch on this device
  uint64_t* twiddles = nullptr;   // device address of g_noalloc_twiddles on this device
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_mu;
uint64_t g_host_twiddles[2 * sg::kTwDirElems];  // layout of sg::ntt_tables_host
bool g_host_twiddles_ready = false;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// A process-unique id of the calling thread's current context, or 0 when the
// driver cannot give one. A context created after cudaDeviceReset gets a new
// id, and its module holds freshly loaded static arrays (no twiddles), so a
// changed id means the set-up must run again. The two driver calls are reached
// through the runtime's entry-point query: the library links cudart only.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || c == nullptr) return 0;
  if (get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// With the device current: resolve the device addresses of the static arrays
// (host code may not use the symbols' names as pointers) and, the first time
// on a device or whenever its context or the arrays' addresses changed since
// (cudaDeviceReset), fill the twiddle table with a synchronous copy. Resolving
// the addresses runs on every call; it is a table lookup in the runtime.
int setup_device(int dev, DeviceSlot* out) {
  uint64_t* scratch = nullptr;
  uint64_t* tw = nullptr;
  if (cudaGetSymbolAddress((void**)&scratch, g_noalloc_scratch) != cudaSuccess) return SG_ECUDA;
  if (cudaGetSymbolAddress((void**)&tw, g_noalloc_twiddles) != cudaSuccess) return SG_ECUDA;
  const unsigned long long ctx_id = current_context_id();
  std::lock_guard<std::mutex> g(g_mu);
  DeviceSlot& s = g_slots[dev];
  if (!s.ready || s.ctx_id != ctx_id || s.scratch != scratch || s.twiddles != tw) {
    if (!g_host_twiddles_ready) {
      sg::ntt_tables_host(g_host_twiddles);
      g_host_twiddles_ready = true;
    }
    s.ready = false;
    if (cudaMemcpy(tw, g_host_twiddles, sizeof g_host_twiddles, cudaMemcpyHostToDevice) != cudaSuccess)
      return SG_ECUDA;
    s.scratch = scratch;
    s.twiddles = tw;
    s.ctx_id = ctx_id;
    s.ready = true;
  }
  *out = s;
  return SG_OK;
}

// True for device (or managed) memory that belongs to device `dev`. Memory of
// another GPU is refused: without peer access enabled, a kernel that reads it
// faults.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int sg_ntt_noalloc(const uint64_t* d_in, uint64_t* d_out, size_t n_cols, size_t log_n, int inverse,
                              void* cuda_stream) {
  if (!d_in || !d_out || n_cols == 0 || n_cols >= (size_t(1) << 31) || log_n > (size_t)sg::kMaxLogN)
    return SG_EINVAL;
  const size_t n = size_t(1) << log_n;
  if (sg::ntt_scratch_elems(n_cols, (int)log_n) > kNoAllocScratchElems) return SG_ELIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SG_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return SG_EINVAL;
  if (!on_device(d_in, dev) || !on_device(d_out, dev)) return SG_EINVAL;
  DeviceSlot s;
  const int rc = setup_device(dev, &s);
  if (rc != SG_OK) return rc;
  const sg::NttTables t = sg::ntt_tables_view(s.twiddles);
  // Pass 1 writes every scratch element that pass 2 reads, so the scratch left
  // by an earlier call needs no clearing.
  const cudaError_t e = sg::ntt_batch(t, d_in, d_out, (uint32_t)n_cols, n, n, (int)log_n, inverse != 0, n,
                                      log_n > 12 ? s.scratch : nullptr, (cudaStream_t)cuda_stream);
  return e == cudaSuccess ? SG_OK : SG_ECUDA;
}
