// pair_v1.cu -- instantiates the paired velocity kernels of RK stage kind
// 1 (inner stages) for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_v1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<PART_VEL, 1>(pl, m, a, err, s);
}

void attrs_v1() { set_attrs<PART_VEL, 1>(); }

int resident_vel() { return resident_ctas<PART_VEL>(); }
}  // namespace pair
}  // namespace cgfd
