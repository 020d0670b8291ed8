// pair_bs1.cu -- instantiates the paired stress kernels of RK stage kind
// 1 (inner stages) with BF16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_bs1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_STR, 1>(pl, m, a, pl.wk, err, s);
}

void attrs_bs1() { set_attrs<__nv_bfloat16, PART_STR, 1>(); }

int resident_bs() { return resident_ctas<__nv_bfloat16, PART_STR>(); }
void launch_bs1_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_STR, 1, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_bs1_b() { set_attrs<__nv_bfloat16, PART_STR, 1, true>(); }
int resident_bs_b() { return resident_ctas<__nv_bfloat16, PART_STR, true>(); }
}  // namespace pair
}  // namespace cgfd
