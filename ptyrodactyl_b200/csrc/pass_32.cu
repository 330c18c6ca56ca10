// Pass-kernel instantiations for 32x32 grids (N1=4 threads per line, N2=8 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(32, 4, 8)
}  // namespace ptyro
