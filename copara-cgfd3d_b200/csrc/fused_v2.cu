// fused_v2.cu -- instantiates the velocity kernels of RK stage kind 2
// (final stage) for the 8 stencil directions.
#include "stage_fused_impl.cuh"

namespace cgfd {
namespace fused {

void launch_v2(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err,
                  cudaStream_t s) {
  launch_dirs<PART_VEL, 2>(pl, m, a, err, s);
}

void attrs_v2() { set_attrs<PART_VEL, 2>(); }

}  // namespace fused
}  // namespace cgfd
