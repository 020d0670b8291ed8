// stage_pair.cu -- host side of the paired z-marching stage kernels: TMA
// tensor maps, launch plan (persistent grid, z-chunk length) and dispatch.
// The kernels themselves are in stage_pair_impl.cuh, instantiated by
// pair_{v,s}{0,1,2}.cu.
#include "stage_pair_impl.cuh"

#include <new>

namespace cgfd {
namespace pair {
namespace {

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

// 4-D map {x: nx, y: ny, z: nz, component: nc} over float arrays with the
// given pitches (elements), box {bx, by, 1, bc}
bool make_map(CUtensorMap *m, const float *base, int nx, int ny, int nz, int nc, size_t pitch_y,
              size_t pitch_z, size_t pitch_c, int bx, int by, int bc) {
  auto fn = encode_fn();
  if (!fn || !base) return false;
  cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nc};
  cuuint64_t strides[3] = {(cuuint64_t)pitch_y * 4, (cuuint64_t)pitch_z * 4,
                           (cuuint64_t)pitch_c * 4};
  cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)bc};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}
// a map over ncomp arrays of the internal field layout
bool field_map(CUtensorMap *m, const Geom &g, const float *base, int ncomp, int bx, int by,
               int bc) {
  return make_map(m, base, g.px, g.nyi, g.nzi, ncomp, g.px, g.plane, g.fstride, bx, by, bc);
}
// a map over one auxiliary set (9 components) of direction d
bool aux_map(CUtensorMap *m, const Geom &g, int d, const float *base, int bc) {
  if (d == 0)
    return make_map(m, base, g.nxa, g.nyi, g.nzi, 9, g.nxa, (size_t)g.nxa * g.nyi, g.astride[0],
                    CX, TY, bc);
  if (d == 1)
    return make_map(m, base, g.px, g.nya, g.nzi, 9, g.px, (size_t)g.px * g.nya, g.astride[1],
                    CX, TY, bc);
  return make_map(m, base, g.px, g.nyi, g.nza, 9, g.px, g.plane, g.astride[2], CX, TY, bc);
}

}  // namespace
}  // namespace pair

using namespace pair;

bool pair_supported(const Geom &g) {
  // tile boxes start on 16-byte boundaries (XO and i0 multiples of 4, px of
  // 32) and the grid is at least one plane deep beyond the stencil reach
  return (XO % 4) == 0 && XO >= 4 && g.px % 32 == 0 && g.nk >= 4;
}

void *pair_create_plan(const Geom &g, float *const sets[4], const float *media,
                       const float *metric, float *const aux[3]) {
  static bool attrs = false;
  if (!attrs) {
    attrs_v0(); attrs_v1(); attrs_v2();
    attrs_s0(); attrs_s1(); attrs_s2();
    attrs = true;
  }
  Plan *pl = new (std::nothrow) Plan();
  if (!pl) return nullptr;
  bool ok = true;
  constexpr int NCV = PartInfo<PART_VEL>::NC, NCS = PartInfo<PART_STR>::NC;
  for (int q = 0; q < 4; ++q) {
    ok = ok && field_map(&pl->haloV[q], g, sets[q], 9, HX, HY, NCV);
    ok = ok && field_map(&pl->haloS[q], g, sets[q], 9, HX, HY, NCS);
    ok = ok && field_map(&pl->ctrV[q], g, sets[q], 9, CX, TY, 3);
    ok = ok && field_map(&pl->ctrT[q], g, sets[q], 9, CX, TY, 6);
  }
  ok = ok && field_map(&pl->coefV, g, media, 3, CX, TY, PartInfo<PART_VEL>::NCOEF);
  ok = ok && field_map(&pl->coefS, g, media, 3, CX, TY, PartInfo<PART_STR>::NCOEF);
  ok = ok && field_map(&pl->met, g, metric, 4, CX, TY, 3);
  for (int d = 0; d < 3; ++d) {
    pl->wk.has_aux[d] = aux[d] != nullptr;
    if (!aux[d]) continue;
    const size_t ss = 9 * g.astride[d];
    for (int t = 0; t < 3; ++t) {  // FA, A, tA
      ok = ok && aux_map(&pl->auxV[d][t], g, d, aux[d] + t * ss, 3);
      ok = ok && aux_map(&pl->auxT[d][t], g, d, aux[d] + t * ss, 6);
    }
  }
  if (!ok) {
    delete pl;
    return nullptr;
  }
  Work &wk = pl->wk;
  wk.ntx = (g.ni + CX - 1) / CX;
  wk.ntiles = wk.ntx * ((g.nj + TY - 1) / TY);
  const int rv = resident_vel(), rs = resident_str();
  const int G = rv < rs ? rv : rs;
  // z-chunk length: minimise (rounds of work over the resident CTAs) x
  // (chunk length + the four window planes read around it)
  double best = 1e30;
  int bestzc = g.nk;
  for (int nzc = 1; nzc <= (g.nk + 7) / 8; ++nzc) {
    const int zc = (g.nk + nzc - 1) / nzc;
    const long items = (long)wk.ntiles * ((g.nk + zc - 1) / zc);
    const long rounds = (items + G - 1) / G;
    const double cost = (double)rounds * (zc + 4);
    if (cost < best - 1e-9) { best = cost; bestzc = zc; }
  }
  wk.zchunk = bestzc;
  wk.nitems = wk.ntiles * ((g.nk + bestzc - 1) / bestzc);
  pl->grid[0] = wk.nitems < rv ? wk.nitems : rv;
  pl->grid[1] = wk.nitems < rs ? wk.nitems : rs;
  return pl;
}

void pair_destroy_plan(void *plan) { delete reinterpret_cast<Plan *>(plan); }

void launch_stage_pair(const void *plan, const StageArgs &a, int in_set, int *err,
                       void *stream) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  cudaStream_t s = (cudaStream_t)stream;
  const int kind = a.rk == 0 ? 0 : (a.rk < 3 ? 1 : 2);
  Maps mv, ms;
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
  for (int d = 0; d < 3; ++d) {
    // prefetched sets: stage input (FA in the first stage, else A), FA, tA
    const int in = (a.rk == 0) ? 0 : 1;
    mv.aux[d][0] = pl.auxV[d][in]; mv.aux[d][1] = pl.auxV[d][0]; mv.aux[d][2] = pl.auxV[d][2];
    ms.aux[d][0] = pl.auxT[d][in]; ms.aux[d][1] = pl.auxT[d][0]; ms.aux[d][2] = pl.auxT[d][2];
  }
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

int pair_plan_info(const void *plan, int *zchunk, int *grid_vel, int *grid_str) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  if (zchunk) *zchunk = pl.wk.zchunk;
  if (grid_vel) *grid_vel = pl.grid[0];
  if (grid_str) *grid_str = pl.grid[1];
  return pl.wk.nitems;
}

}  // namespace cgfd
