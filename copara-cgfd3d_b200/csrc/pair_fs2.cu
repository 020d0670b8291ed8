// pair_fs2.cu -- instantiates the paired stress kernels of RK stage kind
// 2 (final stage) with FP32 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_fs2(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<float, PART_STR, 2>(pl, m, a, pl.wk, err, s);
}

void attrs_fs2() { set_attrs<float, PART_STR, 2>(); }

void launch_fs2_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<float, PART_STR, 2, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_fs2_b() { set_attrs<float, PART_STR, 2, true>(); }
}  // namespace pair
}  // namespace cgfd
