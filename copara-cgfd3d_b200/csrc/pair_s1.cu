// pair_s1.cu -- instantiates the paired stress kernels of RK stage kind
// 1 (inner stages) for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_s1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<PART_STR, 1>(pl, m, a, err, s);
}

void attrs_s1() { set_attrs<PART_STR, 1>(); }

int resident_str() { return resident_ctas<PART_STR>(); }
}  // namespace pair
}  // namespace cgfd
