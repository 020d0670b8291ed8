// pair_hs0.cu -- instantiates the paired stress kernels of RK stage kind
// 0 (first stage) with FP16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_hs0(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__half, PART_STR, 0>(pl, m, a, pl.wk, err, s);
}

void attrs_hs0() { set_attrs<__half, PART_STR, 0>(); }

void launch_hs0_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__half, PART_STR, 0, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_hs0_b() { set_attrs<__half, PART_STR, 0, true>(); }
}  // namespace pair
}  // namespace cgfd
