// pair_fv1.cu -- instantiates the paired velocity kernels of RK stage kind
// 1 (inner stages) with FP32 storage for the 8 stencil directions.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_fv1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<float, PART_VEL, 1>(pl, m, a, err, s);
}

void attrs_fv1() { set_attrs<float, PART_VEL, 1>(); }

int resident_fv() { return resident_ctas<float, PART_VEL>(); }
}  // namespace pair
}  // namespace cgfd
