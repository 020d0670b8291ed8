// pair_hs1.cu -- instantiates the paired stress kernels of RK stage kind
// 1 (inner stages) with FP16 storage for the 8 stencil directions,
// single-model and batched.
#include "stage_pair_impl.cuh"

namespace cgfd {
namespace pair {

void launch_hs1(const Plan &pl, const Maps &m, const StageArgs &a, int *err, cudaStream_t s) {
  launch_dirs<__half, PART_STR, 1>(pl, m, a, pl.wk, err, s);
}

void attrs_hs1() { set_attrs<__half, PART_STR, 1>(); }

int resident_hs() { return resident_ctas<__half, PART_STR>(); }
void launch_hs1_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  launch_dirs<__half, PART_STR, 1, true>(pl, Maps{}, a, wk, err, s);
}

void attrs_hs1_b() { set_attrs<__half, PART_STR, 1, true>(); }
int resident_hs_b() { return resident_ctas<__half, PART_STR, true>(); }
}  // namespace pair
}  // namespace cgfd
