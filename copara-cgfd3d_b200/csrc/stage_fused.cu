// stage_fused.cu -- z-marching tiled RK stage kernel (placeholder until the
// tiled kernel lands; fused_supported() reports no support so that
// cgfd_create rejects CGFD_KERNEL_FUSED instead of running anything else).
#include "cgfd_internal.cuh"

namespace cgfd {

bool fused_supported(const Geom &) { return false; }

void launch_stage_fused(const StageArgs &, void *) {}

}  // namespace cgfd
