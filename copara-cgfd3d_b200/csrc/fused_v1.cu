// fused_v1.cu -- instantiates the velocity kernels of RK stage kind 1
// (inner stages) for the 8 stencil directions.
#include "stage_fused_impl.cuh"

namespace cgfd {
namespace fused {

void launch_v1(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err,
                  cudaStream_t s) {
  launch_dirs<PART_VEL, 1>(pl, m, a, err, s);
}

void attrs_v1() { set_attrs<PART_VEL, 1>(); }

int resident_vel() { return resident_ctas<PART_VEL>(); }

}  // namespace fused
}  // namespace cgfd
