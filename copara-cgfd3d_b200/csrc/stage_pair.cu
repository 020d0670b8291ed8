// stage_pair.cu -- host side of the paired z-marching stage kernels: TMA
// tensor maps, launch plan (persistent grid, z-chunk length) and dispatch.
// The kernels themselves are in stage_pair_impl.cuh, instantiated by
// pair_{v,s}{0,1,2}.cu.
#include "stage_pair_impl.cuh"

#include <algorithm>
#include <new>
#include <vector>

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
bool make_map(CUtensorMap *m, const void *base, int nx, int ny, int nz, int nc, size_t pitch_y,
              size_t pitch_z, size_t pitch_c, int bx, int by, int bc, int elem = ELEM_F32) {
  auto fn = encode_fn();
  if (!fn || !base) return false;
  const size_t es_b = elem_size(elem);
  cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nc};
  cuuint64_t strides[3] = {(cuuint64_t)(pitch_y * es_b), (cuuint64_t)(pitch_z * es_b),
                           (cuuint64_t)(pitch_c * es_b)};
  cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)bc};
  cuuint32_t es[4] = {1, 1, 1, 1};
  const CUtensorMapDataType dt = elem == ELEM_F16    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                 : elem == ELEM_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                     : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = fn(m, dt, 4, (void *)base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}
// a map over ncomp arrays of the internal field layout
bool field_map(CUtensorMap *m, const Geom &g, const void *base, int ncomp, int bx, int by,
               int bc, int elem = ELEM_F32) {
  return make_map(m, base, g.px, g.nyi, g.nzi, ncomp, g.px, g.plane, g.fstride, bx, by, bc,
                  elem);
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

#ifndef CGFD_PAIR_ITEMS_PER_CTA
#define CGFD_PAIR_ITEMS_PER_CTA 6
#endif
#ifndef CGFD_PAIR_MIN_CHUNK
#define CGFD_PAIR_MIN_CHUNK 16
#endif
// work list shape: about this many items per resident CTA, z-chunks of at
// least this many planes
constexpr int ITEMS_PER_CTA = CGFD_PAIR_ITEMS_PER_CTA, MIN_CHUNK = CGFD_PAIR_MIN_CHUNK;

bool pair_supported(const Geom &g) {
  // tile boxes start on 16-byte boundaries (XO and i0 multiples of 4, px of
  // 32) and every z-chunk has at least 4 planes
  return (XO % 4) == 0 && XO >= 4 && g.px % 32 == 0 && g.nk >= 4;
}

void *pair_create_plan(const Geom &g, int elem, void *const sets[4], const float *media,
                       const float *metric, float *const aux[3]) {
  static bool attrs = false;
  if (!attrs) {
    attrs_fv0(); attrs_fv1(); attrs_fv2(); attrs_fs0(); attrs_fs1(); attrs_fs2();
    attrs_hv0(); attrs_hv1(); attrs_hv2(); attrs_hs0(); attrs_hs1(); attrs_hs2();
    attrs_bv0(); attrs_bv1(); attrs_bv2(); attrs_bs0(); attrs_bs1(); attrs_bs2();
    attrs = true;
  }
  Plan *pl = new (std::nothrow) Plan();
  if (!pl) return nullptr;
  pl->elem = elem;
  bool ok = true;
  constexpr int NCV = PartInfo<PART_VEL>::NC, NCS = PartInfo<PART_STR>::NC;
  const int hx = (elem == ELEM_F32) ? Halo<float>::HX : Halo<__half>::HX;
  for (int q = 0; q < 4; ++q) {
    ok = ok && field_map(&pl->haloV[q], g, sets[q], 9, hx, HY, NCV, elem);
    ok = ok && field_map(&pl->haloS[q], g, sets[q], 9, hx, HY, NCS, elem);
    ok = ok && field_map(&pl->ctrV[q], g, sets[q], 9, CX, TY, 3, elem);
    ok = ok && field_map(&pl->ctrT[q], g, sets[q], 9, CX, TY, 6, elem);
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
  // work items: the bottom PML layer as a z-chunk of its own, the rest in
  // pieces long enough to amortise the four window planes read around each
  // chunk and numerous enough to balance
  // x tiles start at the grid's first column (a tile whose PML columns share
  // it with interior columns costs about as much per plane as a tile of PML
  // columns alone: the boundary path is latency-bound per plane)
  const int xorg = 0;
  const int ntx = (g.ni - xorg + CX - 1) / CX, nty = (g.nj + TY - 1) / TY;
  const int ntiles = ntx * nty;
  const int rv = elem == ELEM_F16 ? resident_hv() : elem == ELEM_BF16 ? resident_bv()
                                                                    : resident_fv();
  const int rs = elem == ELEM_F16 ? resident_hs() : elem == ELEM_BF16 ? resident_bs()
                                                                    : resident_fs();
  const int G = rv < rs ? rv : rs;
  // (every chunk has at least 4 planes: the kernel's initial issue of four
  // entries relies on it)
  std::vector<int> zb{LFD};
  const int zlo = LFD + g.nabs[4], ztop = g.nk + LFD;
  if (g.nabs[4] >= 8 && ztop - zlo >= 8) zb.push_back(zlo);
  const int zr = zb.back(), rest = ztop - zr;
  int pieces = 1;
  while ((long)ntiles * ((long)zb.size() - 1 + pieces) < (long)ITEMS_PER_CTA * G &&
         rest / (pieces + 1) >= MIN_CHUNK)
    ++pieces;
  for (int q = 1; q <= pieces; ++q) zb.push_back(zr + (int)((long)rest * q / pieces));
  for (size_t c = 0; c + 1 < zb.size(); ++c)
    if (zb[c + 1] - zb[c] < 4) {
      delete pl;
      return nullptr;
    }
  pl->zchunk = (rest + pieces - 1) / pieces;
  // order: the most expensive first (estimated cost: planes x sum over the
  // tile's valid columns of (1 + number of PML directions)), so the cheap
  // items fill the tail; equal costs keep the (z-chunk, tile) order, so
  // neighbouring tiles of a class run together and share halo rows in L2
  struct It { int4 v; double cost; };
  std::vector<It> items;
  for (size_t c = 0; c + 1 < zb.size(); ++c) {
    const bool zp = zb[c] < zlo;
    for (int t = 0; t < ntiles; ++t) {
      const int i0 = xorg + (t % ntx) * CX, j0 = (t / ntx) * TY;
      double w = 0;
      for (int j = j0; j < j0 + TY && j < g.nj; ++j) {
        const bool yp = j < g.nabs[2] || j >= g.nj - g.nabs[3];
        for (int i = i0 < 0 ? 0 : i0; i < i0 + CX && i < g.ni; ++i) {
          const bool xp = i < g.nabs[0] || i >= g.ni - g.nabs[1];
          w += 1 + (xp ? 1 : 0) + (yp ? 1 : 0) + (zp ? 1 : 0);
        }
      }
      items.push_back({make_int4(i0, j0, zb[c], zb[c + 1]), w * (zb[c + 1] - zb[c])});
    }
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const It &x, const It &y) { return x.cost > y.cost; });
  std::vector<int4> hv(items.size());
  for (size_t q = 0; q < items.size(); ++q) hv[q] = items[q].v;
  Work &wk = pl->wk;
  wk.nitems = (int)hv.size();
  int4 *d_items = nullptr;
  int *d_counter = nullptr;
  if (cudaMalloc(&d_items, hv.size() * sizeof(int4)) != cudaSuccess ||
      cudaMemcpy(d_items, hv.data(), hv.size() * sizeof(int4), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMalloc(&d_counter, 2 * sizeof(int)) != cudaSuccess ||
      cudaMemset(d_counter, 0, 2 * sizeof(int)) != cudaSuccess) {
    cudaFree(d_items);
    cudaFree(d_counter);
    delete pl;
    return nullptr;
  }
  wk.items = d_items;
  wk.counter = d_counter;
  pl->grid[0] = wk.nitems < rv ? wk.nitems : rv;
  pl->grid[1] = wk.nitems < rs ? wk.nitems : rs;
  return pl;
}

void pair_destroy_plan(void *plan) {
  Plan *pl = reinterpret_cast<Plan *>(plan);
  if (!pl) return;
  cudaFree((void *)pl->wk.items);
  cudaFree(pl->wk.counter);
  delete pl;
}

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
  // both parts' item counters restart at zero
  cudaMemsetAsync(pl.wk.counter, 0, 2 * sizeof(int), s);
  typedef void (*LaunchFn)(const Plan &, const Maps &, const StageArgs &, int *, cudaStream_t);
  static const LaunchFn fns[3][2][3] = {
      {{launch_fv0, launch_fv1, launch_fv2}, {launch_fs0, launch_fs1, launch_fs2}},
      {{launch_hv0, launch_hv1, launch_hv2}, {launch_hs0, launch_hs1, launch_hs2}},
      {{launch_bv0, launch_bv1, launch_bv2}, {launch_bs0, launch_bs1, launch_bs2}}};
  const int e = pl.elem == ELEM_F16 ? 1 : pl.elem == ELEM_BF16 ? 2 : 0;
  fns[e][0][kind](pl, mv, a, err, s);
  fns[e][1][kind](pl, ms, a, err, s);
  launch_timg(a, s);
}

int pair_plan_info(const void *plan, int *zchunk, int *grid_vel, int *grid_str) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  if (zchunk) *zchunk = pl.zchunk;
  if (grid_vel) *grid_vel = pl.grid[0];
  if (grid_str) *grid_str = pl.grid[1];
  return pl.wk.nitems;
}

}  // namespace cgfd
