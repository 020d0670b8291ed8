// cgfd_internal.cuh -- device data layout and kernel parameter blocks of the
// B200 CGFD solver.
//
// HBM layout (all arrays 256-byte aligned, zero-initialised):
//   * Every wavefield component is a 3-D array with x fastest:
//         idx(ix, iy, iz) = (iz * nyi + iy) * px + ix
//     ix = i_ref + XSH with XSH = XO - 3: the first valid cell sits at
//     XO = 32, so a tile of cells that starts at a valid cell starts on a
//     128-byte line and every warp's 128-byte row of stores covers whole
//     32-byte sectors (no partial-sector writes); iy = j_ref, iz = k_ref.
//     px (x pitch) is a multiple of 32 floats (128 B) and leaves >= 4 zero
//     ghost columns on the right; nyi = nj+6, nzi = nk+6.  Ghost cells are
//     never written, so the one-sided stencils read zeros there exactly like
//     the reference's single-rank run (its ghost planes stay 0).
//   * A field "set" is 9 consecutive components (Vx Vy Vz Txx Tyy Tzz Txy Txz
//     Tyz) separated by fstride elements.  The solver keeps 4 sets: FW (step
//     start), Wa and Wb (stage outputs, ping-pong because the stencil cannot
//     run in place) and tW (RK accumulator).
//   * ADE CFS-PML auxiliaries are compact per direction:
//         X: (iz * nyi + iy) * nxa + xa      xa = i (left layer) or
//            i - (ni - nabs1) + xaoff (right layer); xaoff >= nabs0 is chosen
//            congruent to ni - nabs1 modulo 4 so that xa and i agree modulo
//            4 (aligned pair and tile accesses) and nxa is a multiple of 4
//         Y: (iz * nya + ya) * px  + ix      ya in [0, nabs2+nabs3)
//         Z: (za * nyi + iy) * px  + ix      za in [0, nabs4+nabs5)
//     each with 3 sets (FA step start, A stage value updated in place since
//     the auxiliaries are read only at their own cell, tA accumulator).
//   * Media are stored as (lambda+2mu, mu, 1/rho); the metric as zeta_x,
//     zeta_y, zeta_z, jac; 1-D PML profiles APD, B, DB per axis in the same
//     internal index space; the free-surface matrices matVx2Vz / matVy2Vz as
//     18 planes of px*nyi.
#pragma once

#include <cstddef>
#include <cstdint>

#include <vector_types.h>

#include "elem.cuh"

namespace cgfd {

constexpr int LFD = 3;   // ghost width of the reference (LenFD)
#ifndef CGFD_XO
#define CGFD_XO 32
#endif
constexpr int XO = CGFD_XO;  // internal x index of the first valid cell
constexpr int XSH = XO - LFD;  // internal x index = reference x index + XSH
constexpr int NCOMP = 9;

enum { VX = 0, VY, VZ, TXX, TYY, TZZ, TXY, TXZ, TYZ };

// DRP/opt MacCormack one-sided operator (Zhang 2006; the reference's
// src/typenew.h:52-56), Gottlieb 2-4 (typenew.h:69-71).
#define CGFD_DA_1 (-0.30874f)
#define CGFD_DA0 (-0.6326f)
#define CGFD_DA1 (1.23300f)
#define CGFD_DA2 (-0.3334f)
#define CGFD_DA3 (0.04168f)
#define CGFD_MA0 (-1.1666666666666667f)
#define CGFD_MA1 (1.3333333333333333f)
#define CGFD_MA2 (-0.16666666666666666f)

struct Geom {
  int ni, nj, nk;      // valid cells
  int px, nyi, nzi;    // internal dims (px = x pitch)
  int top;             // iz of the free surface (nk + 2)
  int con;             // ConIndex (iz)
  int nabs[6];
  int nxa, nya, nza;   // auxiliary widths per direction (nxa: row pitch)
  int xaoff;           // X auxiliaries: xa of the first right-hand PML column
  size_t plane;        // px * nyi
  size_t fstride;      // elements between components of a set
  size_t astride[3];   // elements between components of an aux set
  // components per aux set: 9 (one per field), or 6 for the paired kernels:
  // V's three, then one per velocity derivative in that direction, from
  // which the six stresses' auxiliaries follow linearly
  int ncaux;
};

__host__ __device__ inline size_t gidx(const Geom &g, int ix, int iy, int iz) {
  return ((size_t)iz * g.nyi + iy) * g.px + ix;
}

// Arguments of one RK stage (RKite + Iteration*), for any kernel family.
struct StageArgs {
  Geom g;
  int rk;              // 0..3
  int X, Y, Z;         // +1 forward / -1 backward per axis
  float h;             // steph
  float adt, bdt;      // RK4A[rk]*dt (0 for rk 3), RK4B[rk]*dt
  // tW elision (the paired kernels, their traction image and sources): the
  // first stage writes no tW; the second rebuilds it from FW and the first
  // stage's output as FW + rtw * (W - FW), rtw = RK4B[0]/RK4A[0], which
  // equals FW + RK4B[0]*dt*RHS because W = FW + RK4A[0]*dt*RHS.  (The ADE
  // auxiliaries keep their tA: rebuilding it would hold the stage input's
  // auxiliaries in registers up to the update, which cost more in the
  // latency-bound PML tiles than the bytes saved.)
  bool tw_skip;
  float rtw;
  // field sets, of the storage element type elem (ELEM_F32 / F16 / BF16)
  const void *in;      // stencil input set (FW for rk 0, else previous W)
  const void *fw;      // FW (rk 1,2 read it)
  void *out;           // output set: W (rk 0..2) or FW (rk 3)
  void *tw;            // tW
  int elem;
  float sc[NCOMP];     // value of one stored unit per component (2^k)
  float isc[NCOMP];    // its inverse (stored units per value)
  const float *lam2mu, *mu, *irho;
  const float *zx, *zy, *zz, *jac;
  // planes iz < zu_end (<= ConIndex) have one zeta_z on every valid cell,
  // zzp[iz]: the tiled kernels skip their metric tiles (zeta_x, zeta_y are
  // not used below ConIndex)
  const float *zzp;
  int zu_end;
  bool flat;           // metric is zeta=(0,0,1), jac=1 everywhere
  bool plain_interior; // B = 1 and DB = APD = 0 outside the PML layers
  const float *matv;   // 18 planes: matVx2Vz[0..8], matVy2Vz[0..8]
  const float *apd[3], *b[3], *db[3];
  // aux sets per direction: ain (FA for rk 0 else A), afw (FA), aout (A, or
  // FA for rk 3), tA; null when that direction has no PML
  const float *ain[3];
  const float *afw[3];
  float *aout[3];
  float *ta[3];
};

// Point sources, applied after a stage as W_out += adt*S, tW += bdt*S
// (the update is linear in the RHS, so this equals adding S to hW first).
struct SourceArgs {
  Geom g;
  int nmnt, nfrc;
  const int *mcell;    // internal linear index of each moment source
  const float *mcoef;  // 6 per source: M / (h^3 J)
  const float *mstf;   // nmnt * nstfm
  int nstfm;
  const int *fcell;
  const float *fcoef;  // 3 per source: f / (h^3 J rho) (x2 on the surface)
  const float *fstf;
  int nstff;
  int tinc;            // 0, 1, 1, 2 by stage
  int tindex;          // >= 0: use it; < 0: 2*(*step)+tinc
  const int *step;     // device step counter
  float adt, bdt;
  bool tw_skip;        // first stage: tW is not written (see StageArgs)
  void *out, *tw;      // field sets of element type elem
  int elem;
  float isc[NCOMP];
  int rk;
  // focal points (cgfd_upload_focal): cells, series [6][nfoc][fnt]
  int nfoc, fnt;
  const int *foccell;
  const float *focmom;
  float fdt, dt, h;
  const float *jac;
  // source smoothing (cgfd_set_source_smoothing): kinds spread over 7^3
  // nodes (bit 0 moments, 1 forces, 2 focal points) are left out of the
  // point kernels and added by the spread list: nsp cells, the entries of
  // cell u at [spoff[u], spoff[u+1]), each a source row (kind << 28 | q)
  // and 6 coefficients
  unsigned smooth;
  int nsp;
  const int *spcell, *spoff, *sprow;
  const float *spcoef;
};

void launch_stage_simple(const StageArgs &a, void *stream);
// text returned by cgfd_last_error(NULL, ...)
void set_global_error(const char *msg);
// traction-image velocity update of the top 3 layers (after the fused kernels)
void launch_timg(const StageArgs &a, void *stream);
bool fused_supported(const Geom &g);
// Tensor maps and launch shape of the fused kernels for one solver's buffers
// (sets = FW, Wa, Wb, tW).  nullptr when a tensor map cannot be encoded.
void *fused_create_plan(const Geom &g, float *const sets[4], const float *media,
                        const float *metric);
void fused_destroy_plan(void *plan);
// Both kernels (velocity, stress) of one RK stage; in_set is 0 (FW), 1 or 2.
void launch_stage_fused(const void *plan, const StageArgs &a, int in_set, int *err,
                        void *stream);
int fused_plan_info(const void *plan, int *zchunk, int *grid_vel, int *grid_str);
// The paired kernels (two x-adjacent cells per thread, stage_pair.cu); aux
// holds the three directions' auxiliary arrays (null: no PML there).
// Shape of the paired kernels' work list (the autotuner's knobs): about
// items_per_cta items per resident CTA, z-chunks of at least min_chunk
// planes, PML columns weighted (1 + pml_weight per direction) in the cost
// order.
#ifndef CGFD_TAIL_CHUNK
#define CGFD_TAIL_CHUNK 8
#endif
struct WorkParams {
  int items_per_cta = 6;
  int min_chunk = 16;
  double pml_weight = 1.0;
  // the last G items (one per resident CTA) are cut into chunks of about
  // this many planes, so that the launch ends on short items (0: no cut)
  int tail_chunk = CGFD_TAIL_CHUNK;
};
bool pair_supported(const Geom &g);
bool pair_set_work(void *plan, const WorkParams &wp);
// test hook (cgfd_test_withhold_copy): every wait of the plan's kernels gives
// up after wait_s, and with withhold >= 0 the velocity part's CTA 0 does not
// issue the halo copy of entry `withhold` of its first item; withhold < 0
// restores the defaults
bool pair_set_wait_test(void *plan, double wait_s, int withhold);
WorkParams pair_get_work(const void *plan);
void *pair_create_plan(const Geom &g, int elem, void *const sets[4], const float *media,
                       const float *metric, float *const aux[3]);
void pair_destroy_plan(void *plan);
// a second stream and two events (cudaStream_t / cudaEvent_t) for work
// that may run beside the stage kernels
struct SideStream {
  void *stream, *fork, *join;
  void *stream2, *fork2, *join2;  // the stress part beside the velocity part
};
// the paired kernels run with a.tw_skip set (tW elision); with side, the
// traction image runs on side->stream and the stress part on side->stream2,
// beside the velocity part (the three read only the stage input and write
// disjoint components)
void launch_stage_pair(const void *plan, const StageArgs &a, int in_set, int *err, void *stream,
                       const SideStream *side = nullptr);
int pair_plan_info(const void *plan, int *zchunk, int *grid_vel, int *grid_str);
// A batch of models (one storage type) in one persistent launch per stage
// part: per-model buffers as n x 4 sets, n media, n metrics, n x 3
// auxiliaries.
void *pair_create_batch_plan(int n, const Geom *gs, void *const *sets, const float *const *media,
                             const float *const *metric, float *const *aux, int elem);
// the models' stage arguments, [pattern * 4 + stage][model]
bool pair_batch_set_args(void *plan, const StageArgs *args);
// both parts and the traction image of stage rep.rk (step pattern `pattern`)
// for every model; rep carries the stage's X, Y, Z and rk
void launch_stage_pair_batch(const void *plan, int pattern, const StageArgs &rep, int *err,
                             void *stream);
// learned absorbing layer (mlp.cu): the correction of every layer cell
// (gain: [depth][9]; delta: 9 x n scratch), and the training features of
// the layer's cells
// fw: FW of element type elem, sc: its per-component scales (stored value
// times sc is the value)
struct ScaleSet {
  float sc[NCOMP];
};
size_t mlp_delta_smem();
void mlp_set_attrs();
void launch_mlp_step(const void *fw, int elem, size_t fs, const ScaleSet &sc, const float *lam2mu,
                     const float *irho, const int4 *cells, int n, const void *w, const float *gain,
                     int width, float *delta, void *stream);
void launch_mlp_features(const void *fw, int elem, size_t fs, const ScaleSet &sc,
                         const float *lam2mu, const float *irho, const int4 *cells, int n,
                         float *xs, float *scales, float *zs, void *stream);
// the traction image of n models (args: device array, one per model)
void launch_timg_batch(const StageArgs *args, int n, int max_ni, int max_nj, int elem,
                       void *stream);

}  // namespace cgfd
