// Pass-kernel instantiations for 16x16 grids (N1=4 threads per line, N2=4 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(16, 4, 4)
}  // namespace ptyro
