// fused_s2.cu -- instantiates the stress kernels of RK stage kind 2
// (final stage) for the 8 stencil directions.
#include "stage_fused_impl.cuh"

namespace cgfd {
namespace fused {

void launch_s2(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err,
                  cudaStream_t s) {
  launch_dirs<PART_STR, 2>(pl, m, a, err, s);
}

void attrs_s2() { set_attrs<PART_STR, 2>(); }

}  // namespace fused
}  // namespace cgfd
