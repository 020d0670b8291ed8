// pair_hv1.cu -- instantiates the paired velocity kernels of RK stage kind
// 1 (inner stages) with FP16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_hv1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__half, PART_VEL, 1>(pl, m, a, pl.wk, err, s);
}

void attrs_hv1() { set_attrs<__half, PART_VEL, 1>(); }

int resident_hv() { return resident_ctas<__half, PART_VEL>(); }
void launch_hv1_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__half, PART_VEL, 1, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_hv1_b() { set_attrs<__half, PART_VEL, 1, true>(); }
int resident_hv_b() { return resident_ctas<__half, PART_VEL, true>(); }
}  // namespace pair
}  // namespace cgfd
