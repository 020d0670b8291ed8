// pair_bs2.cu -- instantiates the paired stress kernels of RK stage kind
// 2 (final stage) with BF16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_bs2(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_STR, 2>(pl, m, a, pl.wk, err, s);
}

void attrs_bs2() { set_attrs<__nv_bfloat16, PART_STR, 2>(); }

void launch_bs2_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_STR, 2, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_bs2_b() { set_attrs<__nv_bfloat16, PART_STR, 2, true>(); }
}  // namespace pair
}  // namespace cgfd
