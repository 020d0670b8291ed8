// pair_fs1.cu -- instantiates the paired stress kernels of RK stage kind
// 1 (inner stages) with FP32 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_fs1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<float, PART_STR, 1>(pl, m, a, pl.wk, err, s);
}

void attrs_fs1() { set_attrs<float, PART_STR, 1>(); }

int resident_fs() { return resident_ctas<float, PART_STR>(); }
void launch_fs1_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<float, PART_STR, 1, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_fs1_b() { set_attrs<float, PART_STR, 1, true>(); }
int resident_fs_b() { return resident_ctas<float, PART_STR, true>(); }
}  // namespace pair
}  // namespace cgfd
