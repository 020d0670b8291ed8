// stage_fused.cu -- host side of the fused z-marching stage kernels: TMA
// tensor maps, launch plan (persistent grid, z-chunk length) and dispatch.
// The kernels themselves are in stage_fused_impl.cuh, instantiated by
// fused_{v,s}{0,1,2}.cu.
#include "stage_fused_impl.cuh"

#include <new>

namespace cgfd {
namespace fused {
namespace {

#ifndef CGFD_L2_PROMO
#define CGFD_L2_PROMO CU_TENSOR_MAP_L2_PROMOTION_L2_128B
#endif
constexpr CUtensorMapL2promotion L2_PROMO = CGFD_L2_PROMO;

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 4-D map over ncomp arrays of the internal layout: {x: px, y: nyi, z: nzi,
// component}, with a box of {bx, by, 1, bc}
bool make_map(CUtensorMap *m, const Geom &g, const float *base, int ncomp, int bx, int by,
              int bc) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)g.px, (cuuint64_t)g.nyi, (cuuint64_t)g.nzi,
                        (cuuint64_t)ncomp};
  cuuint64_t strides[3] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.plane * 4,
                           (cuuint64_t)g.fstride * 4};
  cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)bc};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  L2_PROMO, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace
}  // namespace fused

using namespace fused;

bool fused_supported(const Geom &g) {
  // tile boxes start on 16-byte boundaries (XO = 4 floats, px a multiple of
  // 32) and the grid is at least one plane deep beyond the stencil reach
  return (XO % 4) == 0 && g.px % 32 == 0 && g.nk >= 4;
}

void *fused_create_plan(const Geom &g, float *const sets[4], const float *media,
                        const float *metric) {
  static bool attrs = false;
  if (!attrs) {
    attrs_v0(); attrs_v1(); attrs_v2();
    attrs_s0(); attrs_s1(); attrs_s2();
    attrs = true;
  }
  Plan *pl = new (std::nothrow) Plan();
  if (!pl) return nullptr;
  bool ok = true;
  for (int q = 0; q < 4; ++q) {
    ok = ok && make_map(&pl->haloV[q], g, sets[q], 9, BOXX, BOXY, PartInfo<PART_VEL>::NC);
    ok = ok && make_map(&pl->haloS[q], g, sets[q], 9, BOXX, BOXY, PartInfo<PART_STR>::NC);
    ok = ok && make_map(&pl->ctrV[q], g, sets[q], 9, TX, TY, PartInfo<PART_VEL>::NS);
    ok = ok && make_map(&pl->ctrT[q], g, sets[q], 9, TX, TY, PartInfo<PART_STR>::NS);
  }
  ok = ok && make_map(&pl->coefV, g, media, 3, TX, TY, PartInfo<PART_VEL>::NCOEF);
  ok = ok && make_map(&pl->coefS, g, media, 3, TX, TY, PartInfo<PART_STR>::NCOEF);
  ok = ok && make_map(&pl->met, g, metric, 4, TX, TY, 3);
  if (!ok) {
    delete pl;
    return nullptr;
  }
  pl->ntx = (g.ni + TX - 1) / TX;
  pl->ntiles = pl->ntx * ((g.nj + TY - 1) / TY);
  const int G = resident_vel() < resident_str() ? resident_vel()
                                                                     : resident_str();
  // z-chunk length: minimise (rounds of work over the resident CTAs) x
  // (chunk length + start-up planes)
  double best = 1e30;
  int bestzc = g.nk;
  for (int nzc = 1; nzc <= (g.nk + 7) / 8; ++nzc) {
    const int zc = (g.nk + nzc - 1) / nzc;
    const long items = (long)pl->ntiles * ((g.nk + zc - 1) / zc);
    const long rounds = (items + G - 1) / G;
    const double cost = (double)rounds * (zc + 6);
    if (cost < best - 1e-9) { best = cost; bestzc = zc; }
  }
  pl->zchunk = bestzc;
  pl->nitems = pl->ntiles * ((g.nk + bestzc - 1) / bestzc);
  pl->grid[0] = pl->nitems < resident_vel() ? pl->nitems : resident_vel();
  pl->grid[1] = pl->nitems < resident_str() ? pl->nitems : resident_str();
  return pl;
}

void fused_destroy_plan(void *plan) { delete reinterpret_cast<Plan *>(plan); }

void launch_stage_fused(const void *plan, const StageArgs &a, int in_set, int *err,
                        void *stream) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  cudaStream_t s = (cudaStream_t)stream;
  const int kind = a.rk == 0 ? 0 : (a.rk < 3 ? 1 : 2);
  StageMaps mv, ms;
  mv.halo = pl.haloV[in_set];
  mv.u0 = kind == 2 ? pl.ctrV[3] : pl.ctrV[0];
  mv.u1 = pl.ctrV[3];
  mv.coef = pl.coefV;
  mv.met = pl.met;
  ms.halo = pl.haloS[in_set];
  ms.u0 = kind == 2 ? pl.ctrT[3] : pl.ctrT[0];
  ms.u1 = pl.ctrT[3];
  ms.coef = pl.coefS;
  ms.met = pl.met;
  if (kind == 0) {
    launch_v0(pl, mv, a, err, s);
    launch_s0(pl, ms, a, err, s);
  } else if (kind == 1) {
    launch_v1(pl, mv, a, err, s);
    launch_s1(pl, ms, a, err, s);
  } else {
    launch_v2(pl, mv, a, err, s);
    launch_s2(pl, ms, a, err, s);
  }
  launch_timg(a, s);
}

int fused_plan_info(const void *plan, int *zchunk, int *grid_vel, int *grid_str) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  if (zchunk) *zchunk = pl.zchunk;
  if (grid_vel) *grid_vel = pl.grid[0];
  if (grid_str) *grid_str = pl.grid[1];
  return pl.nitems;
}

}  // namespace cgfd
