// pair_s0.cu -- instantiates the paired stress kernels of RK stage kind
// 0 (first stage) for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_s0(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<PART_STR, 0>(pl, m, a, err, s);
}

void attrs_s0() { set_attrs<PART_STR, 0>(); }

}  // namespace pair
}  // namespace cgfd
