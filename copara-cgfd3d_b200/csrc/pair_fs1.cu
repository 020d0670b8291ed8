// pair_fs1.cu -- instantiates the paired stress kernels of RK stage kind
// 1 (inner stages) with FP32 storage for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_fs1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<float, PART_STR, 1>(pl, m, a, err, s);
}

void attrs_fs1() { set_attrs<float, PART_STR, 1>(); }

int resident_fs() { return resident_ctas<float, PART_STR>(); }
}  // namespace pair
}  // namespace cgfd
