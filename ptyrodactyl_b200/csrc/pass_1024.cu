// Pass-kernel instantiations for 1024x1024 grids (N1=32 threads per line, N2=32 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(1024, 32, 32)
}  // namespace ptyro
