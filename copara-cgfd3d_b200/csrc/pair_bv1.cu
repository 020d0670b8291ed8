// pair_bv1.cu -- instantiates the paired velocity kernels of RK stage kind
// 1 (inner stages) with BF16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_bv1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_VEL, 1>(pl, m, a, pl.wk, err, s);
}

void attrs_bv1() { set_attrs<__nv_bfloat16, PART_VEL, 1>(); }

int resident_bv() { return resident_ctas<__nv_bfloat16, PART_VEL>(); }
void launch_bv1_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__nv_bfloat16, PART_VEL, 1, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_bv1_b() { set_attrs<__nv_bfloat16, PART_VEL, 1, true>(); }
int resident_bv_b() { return resident_ctas<__nv_bfloat16, PART_VEL, true>(); }
}  // namespace pair
}  // namespace cgfd
