// Pass-kernel instantiations for 256x256 grids (N1=16 threads per line, N2=16 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(256, 16, 16)

// TMA completion waits of this unit's paired column passes that hit their poll
// limit, on the current device (0 when every copy completed).
unsigned int pair_wait_timeouts_256() {
  unsigned int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_pair_wait_timeouts, sizeof v) != cudaSuccess) return 0xffffffffu;
  return v;
}
}  // namespace ptyro
