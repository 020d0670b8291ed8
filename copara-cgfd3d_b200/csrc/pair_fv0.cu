// pair_fv0.cu -- instantiates the paired velocity kernels of RK stage kind
// 0 (first stage) with FP32 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_fv0(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<float, PART_VEL, 0>(pl, m, a, pl.wk, err, s);
}

void attrs_fv0() { set_attrs<float, PART_VEL, 0>(); }

void launch_fv0_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<float, PART_VEL, 0, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_fv0_b() { set_attrs<float, PART_VEL, 0, true>(); }
}  // namespace pair
}  // namespace cgfd
