// fused_v0.cu -- instantiates the velocity kernels of RK stage kind 0
// (first stage) for the 8 stencil directions.
#include "stage_fused_impl.cuh"

namespace cgfd {
namespace fused {

void launch_v0(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err,
                  cudaStream_t s) {
  launch_dirs<PART_VEL, 0>(pl, m, a, err, s);
}

void attrs_v0() { set_attrs<PART_VEL, 0>(); }

}  // namespace fused
}  // namespace cgfd
