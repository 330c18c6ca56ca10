// Forward model for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory and give a custom call no way to
// allocate or to ask for a workspace: an XLA FFI handler registered without a
// workspace operand, code that runs while a CUDA graph is being captured (where
// cudaMalloc is not allowed), or a plugin host with a fixed memory budget. For
// them ptyro_ms_forward_noalloc runs the same batched forward as ptyro_ms_forward
// with its scratch in a fixed array that lives in this library's device image.
//
// Rules of use:
// * The scratch is kPtyroStaticScratchBytes (64 MiB) per GPU. Every GPU on which
//   this library's device code is loaded holds it until the process exits.
// * Each call looks up the array's device address (cudaGetSymbolAddress, with the
//   calling device current) unless its stream is being captured; a captured call
//   uses the address the last uncaptured call on that device found. Make one call on
//   each device before any stream capture begins. (Looking the address up again
//   keeps it right after cudaDeviceReset, which reloads the module.)
// * All calls on a device share the one array and it keeps whatever the last
//   call left there. Nothing in it has to start at zero: the forward writes every
//   region (twiddles, propagator, transmission table, probe spectrum, ramps,
//   wave slots) before it reads it. Calls whose work overlaps on the GPU (two
//   streams, or two host threads) race on the array and give wrong results;
//   serialise them on one stream.
// * The batch is the largest that fits. If not even one probe fits with the
//   optional interleaved transmission tables of the default variant (tune bit
//   16384: two more tables of 8 bytes per pixel and slice), the tables are left
//   out (same results, bit for bit) and the batch is searched again; a job whose
//   smallest layout still does not fit is rejected with PTYRO_ERR_WORKSPACE before
//   anything is launched.
// * The call cannot hand back the device status word (the first word of the array,
//   see PTYRO_WS_STATUS_BYTES), so when a bounded wait inside the forward gave up,
//   a last kernel fills `patterns` with NaN: failed results never look valid.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/ptyro_b200.h"

namespace ptyro {

constexpr size_t kPtyroStaticScratchBytes = (size_t)PTYRO_STATIC_SCRATCH_BYTES;

// Sets the message ptyro_last_error() returns (defined with it in ms_engine.cu).
void set_error_message(const std::string& msg);

// Host code sees only a stand-in for this symbol; its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_static_scratch[kPtyroStaticScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

int scratch_for_current_device(cudaStream_t st, void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error_message(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return PTYRO_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error_message("device ordinal out of range for the static scratch table");
    return PTYRO_ERR_INVALID;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) {
    set_error_message(std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    return PTYRO_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (cap == cudaStreamCaptureStatusNone || !g_scratch_ptr[dev]) {
    if (cap != cudaStreamCaptureStatusNone) {
      set_error_message("the no-alloc forward's first call on a device must not be captured");
      return PTYRO_ERR_INVALID;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error_message(std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
      return PTYRO_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return PTYRO_OK;
}

// NaN into every pattern value when the forward's status word is set.
__global__ void k_nan_if_failed(const unsigned int* status, float* patterns, size_t count) {
  if (*status == 0u) return;
  const float nan = __int_as_float(0x7fc00000);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    patterns[i] = nan;
}

// The largest batch (<= want) whose layout fits the static scratch, or 0.
int largest_batch(ptyro_ms_params* q, int want) {
  int lo = 0, hi = want;
  while (lo < hi) {
    const int mid = lo + (hi - lo + 1) / 2;
    q->batch = mid;
    if (ptyro_ms_workspace_bytes(q) <= kPtyroStaticScratchBytes) lo = mid; else hi = mid - 1;
  }
  return lo;
}
}  // namespace
}  // namespace ptyro

extern "C" {

int ptyro_ms_forward_noalloc(const ptyro_ms_params* p, const float* potential, const float* modes,
                             const float* weights, const double* positions, float* patterns, void* stream) {
  using namespace ptyro;
  if (!p) {
    set_error_message("params is NULL");
    return PTYRO_ERR_INVALID;
  }
  ptyro_ms_params q = *p;
  if (ptyro_ms_workspace_bytes(&q) == 0) {  // invalid geometry: let the forward report why
    return ptyro_ms_forward(&q, potential, modes, weights, positions, patterns, nullptr, 0, stream);
  }
  if (q.num_probes == 0) return PTYRO_OK;
  // the largest batch whose layout fits the static scratch; without the optional
  // interleaved transmission tables if not even one probe fits with them
  const int want = q.batch > 0 ? q.batch : (q.num_probes > 0 ? q.num_probes : 1);
  int lo = largest_batch(&q, want);
  if (lo == 0 && (q.tune & 16384)) {
    q.tune &= ~16384;
    lo = largest_batch(&q, want);
  }
  if (lo == 0 || (p->batch > 0 && lo < p->batch)) {
    q.batch = p->batch > 0 ? p->batch : 1;
    set_error_message("job needs " + std::to_string(ptyro_ms_workspace_bytes(&q)) +
                      " bytes of scratch but the no-alloc forward has a fixed " +
                      std::to_string(kPtyroStaticScratchBytes) +
                      " bytes; use ptyro_ms_forward with a caller-provided workspace");
    return PTYRO_ERR_WORKSPACE;
  }
  q.batch = lo;
  void* scratch = nullptr;
  int rc = scratch_for_current_device((cudaStream_t)stream, &scratch);
  if (rc) return rc;
  rc = ptyro_ms_forward(&q, potential, modes, weights, positions, patterns, scratch, kPtyroStaticScratchBytes,
                        stream);
  if (rc) return rc;
  const size_t count = (size_t)q.num_probes * q.n * q.n;
  k_nan_if_failed<<<148 * 4, 256, 0, (cudaStream_t)stream>>>((const unsigned int*)scratch, patterns, count);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error_message(std::string("k_nan_if_failed: ") + cudaGetErrorString(e));
    return PTYRO_ERR_CUDA;
  }
  return PTYRO_OK;
}

}  // extern "C"
