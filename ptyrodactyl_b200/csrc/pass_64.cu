// Pass-kernel instantiations for 64x64 grids (N1=8 threads per line, N2=8 points per thread).
#include "pass_launch.cuh"

namespace ptyro {
PTYRO_DEFINE_PASS_LAUNCHER(64, 8, 8)
}  // namespace ptyro
