// Pass-kernel instantiations for 512x512 grids (N1=16 threads per line, N2=32 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(512, 16, 32)
}  // namespace ptyro
