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
    return make_map(m, base, g.nxa, g.nyi, g.nzi, g.ncaux, g.nxa, (size_t)g.nxa * g.nyi, g.astride[0],
                    CX, TY, bc);
  if (d == 1)
    return make_map(m, base, g.px, g.nya, g.nzi, g.ncaux, g.px, (size_t)g.px * g.nya, g.astride[1],
                    CX, TY, bc);
  return make_map(m, base, g.px, g.nyi, g.nza, g.ncaux, g.px, g.plane, g.astride[2], CX, TY, bc);
}

}  // namespace
}  // namespace pair

using namespace pair;

bool pair_supported(const Geom &g) {
  // tile boxes start on 16-byte boundaries (XO and i0 multiples of 4, px of
  // 32) and every z-chunk has at least 4 planes
  return (XO % 4) == 0 && XO >= 4 && g.px % 32 == 0 && g.nk >= 4;
}

namespace pair {
namespace {

void set_all_attrs() {
  static bool done = false;
  if (done) return;
  attrs_fv0(); attrs_fv1(); attrs_fv2(); attrs_fs0(); attrs_fs1(); attrs_fs2();
  attrs_hv0(); attrs_hv1(); attrs_hv2(); attrs_hs0(); attrs_hs1(); attrs_hs2();
  attrs_bv0(); attrs_bv1(); attrs_bv2(); attrs_bs0(); attrs_bs1(); attrs_bs2();
  attrs_fv0_b(); attrs_fv1_b(); attrs_fv2_b(); attrs_fs0_b(); attrs_fs1_b(); attrs_fs2_b();
  attrs_hv0_b(); attrs_hv1_b(); attrs_hv2_b(); attrs_hs0_b(); attrs_hs1_b(); attrs_hs2_b();
  attrs_bv0_b(); attrs_bv1_b(); attrs_bv2_b(); attrs_bs0_b(); attrs_bs1_b(); attrs_bs2_b();
  done = true;
}

// tensor maps of one model's buffers
bool model_maps(ModelMaps *pl, int *has_aux, const Geom &g, int elem, void *const sets[4],
                const float *media, const float *metric, float *const aux[3]) {
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
    has_aux[d] = aux[d] != nullptr;
    if (!aux[d]) continue;
    const size_t ss = (size_t)g.ncaux * g.astride[d];
    for (int t = 0; t < 3; ++t) {  // FA, A, tA
      ok = ok && aux_map(&pl->auxV[d][t], g, d, aux[d] + t * ss, 3);
      ok = ok && aux_map(&pl->auxT[d][t], g, d, aux[d] + t * ss, 3);
    }
  }
  return ok;
}

// the maps of one stage (stage input set, RK kind, stage index) for the
// velocity (mv) and stress (ms) parts
// (rebuild: the second stage under tW elision, whose u1 is the stage input)
// (tw_delta: 16-bit storage, tW kept as tW - FW; the final stage reads FW as
// its first register set and the difference as its second)
void stage_maps(const ModelMaps &pl, int rk, int in_set, bool rebuild, bool tw_delta, Maps &mv,
                Maps &ms) {
  const int kind = rk == 0 ? 0 : (rk < 3 ? 1 : 2);
  const bool fw_first = kind != 2 || tw_delta;
  mv.halo = pl.haloV[in_set];
  mv.u0 = fw_first ? pl.ctrV[0] : pl.ctrV[3];
  mv.u1 = rebuild ? pl.ctrV[in_set] : pl.ctrV[3];
  mv.coef = pl.coefV;
  mv.met = pl.met;
  ms.halo = pl.haloS[in_set];
  ms.u0 = fw_first ? pl.ctrT[0] : pl.ctrT[3];
  ms.u1 = rebuild ? pl.ctrT[in_set] : pl.ctrT[3];
  ms.coef = pl.coefS;
  ms.met = pl.met;
  for (int d = 0; d < 3; ++d) {
    // prefetched sets: stage input (FA in the first stage, else A), FA, tA
    const int in = (rk == 0) ? 0 : 1;
    mv.aux[d][0] = pl.auxV[d][in]; mv.aux[d][1] = pl.auxV[d][0]; mv.aux[d][2] = pl.auxV[d][2];
    ms.aux[d][0] = pl.auxT[d][in]; ms.aux[d][1] = pl.auxT[d][0]; ms.aux[d][2] = pl.auxT[d][2];
  }
}

// x origin of the tile grid (tiles start at i = t * CX - offset).  The
// stage kernels' time follows the number of tile-planes, and a tile that
// touches an x layer runs the slower boundary path for all its columns.
// Candidates 0 and 32 keep every tile row of the field, media and metric
// boxes on a 128-byte boundary (the internal x origin XO is 32); 32 is taken
// when it needs no more tile columns and puts fewer valid columns into tiles
// that touch an x layer (on the 400-wide hill with 20-cell layers: 80
// instead of 144 columns).
int tile_x_offset(const Geom &g) {
  auto ntx = [&](int o) { return (g.ni + o + CX - 1) / CX; };
  auto boundary_cols = [&](int o) {
    int n = 0;
    for (int t = 0; t < ntx(o); ++t) {
      const int i0 = t * CX - o, a = std::max(i0, 0), b = std::min(i0 + CX, g.ni);
      if (a < g.nabs[0] || b > g.ni - g.nabs[1]) n += b - a;
    }
    return n;
  };
  return (ntx(32) == ntx(0) && boundary_cols(32) < boundary_cols(0)) ? 32 : 0;
}

// Work items of one or more models (tile x z-chunk): the bottom PML layer is
// a z-chunk of its own (when it has >= 8 planes), the rest is cut into pieces
// of about len planes (>= MIN_CHUNK; every chunk has >= 4 planes, which the
// kernel's initial issue of four entries relies on).  Order: the most
// expensive first (estimated cost: planes x sum over the tile's valid
// columns of (1 + pml_weight x number of PML directions)), so the cheap
// items fill the tail; equal costs keep the (model, z-chunk, tile) order, so
// neighbouring tiles of a class run together and share halo rows in L2.
std::vector<int4> build_items(const std::vector<Geom> &gs, int G, const WorkParams &wp,
                              int *zchunk) {
  // target chunk length: enough items (items_per_cta per resident CTA) over
  // all models' tile columns
  double colplanes = 0;
  for (const Geom &g : gs)
    colplanes += (double)((g.ni + CX - 1) / CX) * ((g.nj + TY - 1) / TY) * g.nk;
  const double target = (double)wp.items_per_cta * G;
  struct It { int4 v; double cost; };
  std::vector<It> items;
  for (size_t mdl = 0; mdl < gs.size(); ++mdl) {
    const Geom &g = gs[mdl];
    const int xoff = tile_x_offset(g);
    const int ntx = (g.ni + xoff + CX - 1) / CX, nty = (g.nj + TY - 1) / TY;
    const int ntiles = ntx * nty;
    std::vector<int> zb{LFD};
    const int zlo = LFD + g.nabs[4], ztop = g.nk + LFD;
    if (g.nabs[4] >= 8 && ztop - zlo >= 8) zb.push_back(zlo);
    const int zr = zb.back(), rest = ztop - zr;
    int pieces = 1;
    if (gs.size() == 1) {
      while ((long)ntiles * ((long)zb.size() - 1 + pieces) < (long)target &&
             rest / (pieces + 1) >= wp.min_chunk)
        ++pieces;
    } else {
      const double len = colplanes / target > wp.min_chunk ? colplanes / target : wp.min_chunk;
      pieces = (int)(rest / len + 0.5);
      if (pieces < 1) pieces = 1;
      while (pieces > 1 && rest / pieces < 4) --pieces;
    }
    for (int q = 1; q <= pieces; ++q) zb.push_back(zr + (int)((long)rest * q / pieces));
    if (zchunk && mdl == 0) *zchunk = (rest + pieces - 1) / pieces;
    for (size_t c = 0; c + 1 < zb.size(); ++c) {
      if (zb[c + 1] - zb[c] < 4) return {};
      const bool zp = zb[c] < zlo;
      for (int t = 0; t < ntiles; ++t) {
        const int i0 = (t % ntx) * CX - xoff, j0 = (t / ntx) * TY;
        double w = 0;
        for (int j = j0; j < j0 + TY && j < g.nj; ++j) {
          const bool yp = j < g.nabs[2] || j >= g.nj - g.nabs[3];
          for (int i = std::max(i0, 0); i < i0 + CX && i < g.ni; ++i) {
            const bool xp = i < g.nabs[0] || i >= g.ni - g.nabs[1];
            w += 1 + wp.pml_weight * ((xp ? 1 : 0) + (yp ? 1 : 0) + (zp ? 1 : 0));
          }
        }
        items.push_back({make_int4(i0, j0, zb[c] | (zb[c + 1] << 16), (int)mdl),
                         w * (zb[c + 1] - zb[c])});
      }
    }
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const It &x, const It &y) { return x.cost > y.cost; });
  std::vector<int4> hv;
  hv.reserve(items.size());
  // guided end: the last G items (the cheapest) become short chunks, ordered
  // piece by piece (the first piece of every cut item, then the second...)
  // so that CTAs running together stay on neighbouring columns
  size_t ncut = 0;
  if (wp.tail_chunk >= 4) {
    while (ncut < (size_t)G && ncut < items.size()) {
      const int4 v = items[items.size() - 1 - ncut].v;
      if ((v.z >> 16) - (v.z & 0xffff) < 2 * wp.tail_chunk) break;
      ++ncut;
    }
  }
  const size_t keep = items.size() - ncut;
  for (size_t q = 0; q < keep; ++q) hv.push_back(items[q].v);
  std::vector<std::vector<int4>> pieces(ncut);
  size_t maxp = 0;
  for (size_t q = 0; q < ncut; ++q) {
    const int4 v = items[keep + q].v;
    const int z0 = v.z & 0xffff, z1 = v.z >> 16, np = (z1 - z0) / wp.tail_chunk;
    for (int t = 0; t < np; ++t) {
      const int a0 = z0 + (int)((long)(z1 - z0) * t / np);
      const int a1 = z0 + (int)((long)(z1 - z0) * (t + 1) / np);
      pieces[q].push_back(make_int4(v.x, v.y, a0 | (a1 << 16), v.w));
    }
    maxp = std::max(maxp, pieces[q].size());
  }
  for (size_t t = 0; t < maxp; ++t)
    for (size_t q = 0; q < ncut; ++q)
      if (t < pieces[q].size()) hv.push_back(pieces[q][t]);
  return hv;
}

// uploads a work list into the plan (replacing an earlier one)
bool upload_items(Plan *pl, const std::vector<int4> &hv, int rv, int rs) {
  Work &wk = pl->wk;
  if (hv.empty()) return false;
  cudaFree((void *)wk.items);
  wk.items = nullptr;
  int4 *d_items = nullptr;
  if (cudaMalloc(&d_items, hv.size() * sizeof(int4)) != cudaSuccess ||
      cudaMemcpy(d_items, hv.data(), hv.size() * sizeof(int4), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    cudaFree(d_items);
    return false;
  }
  if (!wk.counter) {
    if (cudaMalloc(&wk.counter, 2 * sizeof(int)) != cudaSuccess ||
        cudaMemset(wk.counter, 0, 2 * sizeof(int)) != cudaSuccess)
      return false;
  }
  wk.items = d_items;
  wk.nitems = (int)hv.size();
  pl->grid[0] = wk.nitems < rv ? wk.nitems : rv;
  pl->grid[1] = wk.nitems < rs ? wk.nitems : rs;
  return true;
}

void resident(int elem, bool batch, int *rv, int *rs) {
  if (batch) {
    *rv = elem == ELEM_F16 ? resident_hv_b() : elem == ELEM_BF16 ? resident_bv_b() : resident_fv_b();
    *rs = elem == ELEM_F16 ? resident_hs_b() : elem == ELEM_BF16 ? resident_bs_b() : resident_fs_b();
  } else {
    *rv = elem == ELEM_F16 ? resident_hv() : elem == ELEM_BF16 ? resident_bv() : resident_fv();
    *rs = elem == ELEM_F16 ? resident_hs() : elem == ELEM_BF16 ? resident_bs() : resident_fs();
  }
}

}  // namespace
}  // namespace pair

void *pair_create_plan(const Geom &g, int elem, void *const sets[4], const float *media,
                       const float *metric, float *const aux[3]) {
  set_all_attrs();
  Plan *pl = new (std::nothrow) Plan();
  if (!pl) return nullptr;
  pl->elem = elem;
  pl->geoms.push_back(g);
  pl->mm.resize(1);
  if (!model_maps(&pl->mm[0], pl->wk.has_aux, g, elem, sets, media, metric, aux) ||
      !pair_set_work(pl, WorkParams{})) {
    pair_destroy_plan(pl);
    return nullptr;
  }
  return pl;
}

WorkParams pair_get_work(const void *plan) {
  return reinterpret_cast<const Plan *>(plan)->params;
}

bool pair_set_work(void *plan, const WorkParams &wp) {
  Plan *pl = reinterpret_cast<Plan *>(plan);
  int rv = 0, rs = 0;
  resident(pl->elem, pl->nmodels > 0, &rv, &rs);
  const int G = rv < rs ? rv : rs;
  std::vector<int4> hv = build_items(pl->geoms, G, wp, &pl->zchunk);
  if (!upload_items(pl, hv, rv, rs)) return false;
  pl->params = wp;
  return true;
}

bool pair_set_wait_test(void *plan, double wait_s, int withhold) {
  Plan *pl = reinterpret_cast<Plan *>(plan);
  if (!pl || !(wait_s > 0.0) || wait_s > 60.0) return false;
  pl->wk.wait_us = withhold >= 0 ? (unsigned)(wait_s * 1e6) : ptx::WAIT_US;
  pl->wk.withhold = withhold >= 0 ? withhold : -1;
  return true;
}

void pair_destroy_plan(void *plan) {
  Plan *pl = reinterpret_cast<Plan *>(plan);
  if (!pl) return;
  cudaFree((void *)pl->wk.items);
  cudaFree(pl->wk.counter);
  cudaFree(pl->d_bargs);
  cudaFree(pl->d_bmaps);
  delete pl;
}

void launch_stage_pair(const void *plan, const StageArgs &a, int in_set, int *err, void *stream,
                       const SideStream *side) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  cudaStream_t s = (cudaStream_t)stream;
  const int kind = a.rk == 0 ? 0 : (a.rk < 3 ? 1 : 2);
  Maps mv, ms;
  stage_maps(pl.mm[0], a.rk, in_set, a.tw_skip && a.rk == 1, pl.elem != ELEM_F32, mv, ms);
  // the traction image needs only the stage input and writes what the two
  // parts neither write nor use (the top three layers' V, their tW and x/y
  // auxiliaries): with a side stream it runs beside them, joined at the end
  if (side) {
    cudaEventRecord((cudaEvent_t)side->fork, s);
    cudaStreamWaitEvent((cudaStream_t)side->stream, (cudaEvent_t)side->fork, 0);
    launch_timg(a, side->stream);
    cudaEventRecord((cudaEvent_t)side->join, (cudaStream_t)side->stream);
  }
  // both parts' item counters restart at zero
  cudaMemsetAsync(pl.wk.counter, 0, 2 * sizeof(int), s);
  // the stress part needs the stage input's velocities, not the velocity
  // part's output, and writes other components: with a second side stream
  // its CTAs take the SMs as the velocity part's drain
  cudaStream_t s2 = s;
  if (side && side->stream2) {
    s2 = (cudaStream_t)side->stream2;
    cudaEventRecord((cudaEvent_t)side->fork2, s);
    cudaStreamWaitEvent(s2, (cudaEvent_t)side->fork2, 0);
  }
  typedef void (*LaunchFn)(const Plan &, const Maps &, const StageArgs &, int *, cudaStream_t);
  static const LaunchFn fns[3][2][3] = {
      {{launch_fv0, launch_fv1, launch_fv2}, {launch_fs0, launch_fs1, launch_fs2}},
      {{launch_hv0, launch_hv1, launch_hv2}, {launch_hs0, launch_hs1, launch_hs2}},
      {{launch_bv0, launch_bv1, launch_bv2}, {launch_bs0, launch_bs1, launch_bs2}}};
  const int e = pl.elem == ELEM_F16 ? 1 : pl.elem == ELEM_BF16 ? 2 : 0;
  fns[e][0][kind](pl, mv, a, err, s);
  fns[e][1][kind](pl, ms, a, err, s2);
  if (s2 != s) {
    cudaEventRecord((cudaEvent_t)side->join2, s2);
    cudaStreamWaitEvent(s, (cudaEvent_t)side->join2, 0);
  }
  if (side) cudaStreamWaitEvent(s, (cudaEvent_t)side->join, 0);
  else launch_timg(a, s);
}

// ---------------------------- batched models ------------------------------

void *pair_create_batch_plan(int n, const Geom *gs, void *const *sets, const float *const *media,
                             const float *const *metric, float *const *aux, int elem) {
  set_all_attrs();
  Plan *pl = new (std::nothrow) Plan();
  if (!pl) return nullptr;
  pl->elem = elem;
  pl->nmodels = n;
  pl->geoms.assign(gs, gs + n);
  pl->mm.resize(n);
  bool ok = true;
  for (int i = 0; i < n && ok; ++i) {
    int ha[3];
    ok = model_maps(&pl->mm[i], ha, gs[i], elem, sets + 4 * i, media[i], metric[i],
                    aux + 3 * i);
  }
  // per stage, part and model: the maps of that stage (input set per stage
  // as in the step schedule: FW, Wa, Wb, Wa; batched stages run with tW
  // elision)
  static const int ins[4] = {0, 1, 2, 1};
  std::vector<Maps> hm((size_t)8 * n);
  for (int rk = 0; rk < 4 && ok; ++rk)
    for (int i = 0; i < n; ++i)
      stage_maps(pl->mm[i], rk, ins[rk], rk == 1, elem != ELEM_F32, hm[(size_t)(rk * 2) * n + i],
                 hm[(size_t)(rk * 2 + 1) * n + i]);
  ok = ok && cudaMalloc(&pl->d_bmaps, hm.size() * sizeof(Maps)) == cudaSuccess &&
       cudaMemcpy(pl->d_bmaps, hm.data(), hm.size() * sizeof(Maps), cudaMemcpyHostToDevice) ==
           cudaSuccess &&
       cudaMalloc(&pl->d_bargs, (size_t)16 * n * sizeof(StageArgs)) == cudaSuccess;
  if (!ok || !pair_set_work(pl, WorkParams{})) {
    pair_destroy_plan(pl);
    return nullptr;
  }
  return pl;
}

bool pair_batch_set_args(void *plan, const StageArgs *args) {
  Plan *pl = reinterpret_cast<Plan *>(plan);
  return cudaMemcpy(pl->d_bargs, args, (size_t)16 * pl->nmodels * sizeof(StageArgs),
                    cudaMemcpyHostToDevice) == cudaSuccess;
}

void launch_stage_pair_batch(const void *plan, int pattern, const StageArgs &rep, int *err,
                             void *stream) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  cudaStream_t s = (cudaStream_t)stream;
  const int rk = rep.rk, kind = rk == 0 ? 0 : (rk < 3 ? 1 : 2), n = pl.nmodels;
  Work wv = pl.wk, ws = pl.wk;
  wv.bargs = ws.bargs = pl.d_bargs + (size_t)(pattern * 4 + rk) * n;
  wv.bmaps = pl.d_bmaps + (size_t)(rk * 2) * n;
  ws.bmaps = pl.d_bmaps + (size_t)(rk * 2 + 1) * n;
  typedef void (*LaunchFn)(const Plan &, const StageArgs &, const Work &, int *, cudaStream_t);
  static const LaunchFn fv[3][3] = {{launch_fv0_b, launch_fv1_b, launch_fv2_b},
                                    {launch_hv0_b, launch_hv1_b, launch_hv2_b},
                                    {launch_bv0_b, launch_bv1_b, launch_bv2_b}};
  static const LaunchFn fs[3][3] = {{launch_fs0_b, launch_fs1_b, launch_fs2_b},
                                    {launch_hs0_b, launch_hs1_b, launch_hs2_b},
                                    {launch_bs0_b, launch_bs1_b, launch_bs2_b}};
  const int e = pl.elem == ELEM_F16 ? 1 : pl.elem == ELEM_BF16 ? 2 : 0;
  cudaMemsetAsync(pl.wk.counter, 0, 2 * sizeof(int), s);
  fv[e][kind](pl, rep, wv, err, s);
  fs[e][kind](pl, rep, ws, err, s);
  int mi = 0, mj = 0;
  for (const Geom &g : pl.geoms) {
    mi = g.ni > mi ? g.ni : mi;
    mj = g.nj > mj ? g.nj : mj;
  }
  launch_timg_batch(wv.bargs, n, mi, mj, pl.elem, s);
}

int pair_plan_info(const void *plan, int *zchunk, int *grid_vel, int *grid_str) {
  const Plan &pl = *reinterpret_cast<const Plan *>(plan);
  if (zchunk) *zchunk = pl.zchunk;
  if (grid_vel) *grid_vel = pl.grid[0];
  if (grid_str) *grid_str = pl.grid[1];
  return pl.wk.nitems;
}

}  // namespace cgfd
