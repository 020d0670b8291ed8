// pair_v2.cu -- instantiates the paired velocity kernels of RK stage kind
// 2 (final stage) for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_v2(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<PART_VEL, 2>(pl, m, a, err, s);
}

void attrs_v2() { set_attrs<PART_VEL, 2>(); }

}  // namespace pair
}  // namespace cgfd
