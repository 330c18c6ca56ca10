// Pass-kernel instantiations for 256x256 grids (N1=16 threads per line, N2=16 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(256, 16, 16)
}  // namespace ptyro
