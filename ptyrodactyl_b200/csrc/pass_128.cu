// Pass-kernel instantiations for 128x128 grids (N1=8 threads per line, N2=16 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(128, 8, 16)
}  // namespace ptyro
