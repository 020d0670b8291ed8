// pair_fs0.cu -- instantiates the paired stress kernels of RK stage kind
// 0 (first stage) with FP32 storage for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_fs0(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<float, PART_STR, 0>(pl, m, a, err, s);
}

void attrs_fs0() { set_attrs<float, PART_STR, 0>(); }

}  // namespace pair
}  // namespace cgfd
