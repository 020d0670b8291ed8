// pair_bv0.cu -- instantiates the paired velocity kernels of RK stage kind
// 0 (first stage) with BF16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_bv0(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_VEL, 0>(pl, m, a, pl.wk, err, s);
}

void attrs_bv0() { set_attrs<__nv_bfloat16, PART_VEL, 0>(); }

void launch_bv0_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_VEL, 0, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_bv0_b() { set_attrs<__nv_bfloat16, PART_VEL, 0, true>(); }
}  // namespace pair
}  // namespace cgfd
