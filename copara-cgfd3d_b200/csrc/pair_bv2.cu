// pair_bv2.cu -- instantiates the paired velocity kernels of RK stage kind
// 2 (final stage) with BF16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_bv2(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_VEL, 2>(pl, m, a, pl.wk, err, s);
}

void attrs_bv2() { set_attrs<__nv_bfloat16, PART_VEL, 2>(); }

void launch_bv2_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_VEL, 2, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_bv2_b() { set_attrs<__nv_bfloat16, PART_VEL, 2, true>(); }
}  // namespace pair
}  // namespace cgfd
