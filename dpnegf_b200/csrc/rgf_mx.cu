// Mixed-precision RGF sweep: one instantiation with every feature set (T / DOS / blocks,
// lesser and greater, adjoint), in a translation unit of its own.
#include "rgf_sweep.cuh"

namespace negf {

int rgf_launch_mx(const NegfRgfProblem& p, size_t smem, int grid, cudaStream_t s) {
  return rgf_launch_impl<true, FEAT_ADJOINT>(p, smem, grid, s);
}

}  // namespace negf
