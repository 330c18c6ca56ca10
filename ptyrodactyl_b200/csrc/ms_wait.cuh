// Bounded waits on tile copies (TMA) for the pass kernels, and what a warp does when
// one gives up.
//
// A TMA column pass arms one mbarrier per warp with the byte count of the warp's
// column block, issues the copy, and polls the barrier a bounded number of times.
// If the copy has not landed by then, the warp must not use its shared memory (it is
// stale or still being written) nor write anything back: warp_wait_tile makes that
// decision uniform across the warp (a lane that saw the copy land while another gave
// up still skips), counts the failure, sets PTYRO_STATUS_WAIT_TIMEOUT in the call's
// status word and returns false, and the kernel returns for that warp. No block-wide
// barrier follows the wait in any kernel that uses it, so a warp may leave early.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ptyro_b200.h"

namespace ptyro {

// Polls before a tile wait gives up (each try_wait may itself suspend briefly; the
// whole wait is well under a second).
constexpr int kTileWaitPolls = 1 << 20;

// Waits that gave up in this translation unit's launches, on the current device; read
// on the host by the pass launchers' accessors (ptyro_pass_wait_timeouts).
static __device__ unsigned int g_pair_wait_timeouts = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// true once the barrier's phase `parity` has completed; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Called by all 32 lanes of a warp: true when the tile behind `bar` (phase 0) has
// landed for every lane. Otherwise lane 0 counts the failure and ORs
// PTYRO_STATUS_WAIT_TIMEOUT into *status (if given), and every lane gets false.
__device__ __forceinline__ bool warp_wait_tile(uint32_t bar, int limit, unsigned int* status) {
  const bool ok = __all_sync(0xffffffffu, mbar_wait(bar, 0, limit));
  if (!ok && (threadIdx.x & 31) == 0) {
    atomicAdd(&g_pair_wait_timeouts, 1u);
    if (status) atomicOr(status, PTYRO_STATUS_WAIT_TIMEOUT);
  }
  return ok;
}

}  // namespace ptyro
