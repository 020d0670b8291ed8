// pair_s2.cu -- instantiates the paired stress kernels of RK stage kind
// 2 (final stage) for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_s2(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<PART_STR, 2>(pl, m, a, err, s);
}

void attrs_s2() { set_attrs<PART_STR, 2>(); }

}  // namespace pair
}  // namespace cgfd
