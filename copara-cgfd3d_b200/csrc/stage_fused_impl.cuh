// stage_fused_impl.cuh -- z-marching tiled RK stage kernels for sm_100a
// (templates; instantiated by the fused_*.cu translation units).
//
// One RK stage is two kernels, split along the velocity-stress structure of
// the equations: the velocity part needs only stress derivatives and the
// stress part only velocity derivatives, so each kernel stages only the
// components it differentiates and carries half the register state.
//
// Work is a set of items (a 32 x 4 tile of (x, y) columns times a chunk of
// z-planes); a persistent grid of CTAs walks the items, and each CTA marches
// upwards through its chunk.  Every plane the march needs arrives by TMA
// (cp.async.bulk.tensor, no multicast) into one slot of a 5-slot shared-memory
// ring, on one mbarrier per slot:
//   * the differentiated components of the stage input with an x/y halo (one
//     4-D box {40 x, 10 y, 1 z, NC components}; the one-sided DRP stencils
//     reach -1..+3 or -3..+1 cells, the box covers -4..+4 in x so that its x
//     origin is 16-byte aligned, and -3..+3 in y);
//   * the pointwise operands of the same plane without halo (FW and/or tW
//     components for the RK update, the media coefficients, the metric).
// Loads run 5 planes ahead of the arithmetic, so no warp waits on a plain
// global load during the march; results are written with coalesced stores.
// z stencils run from per-thread register windows of 5 planes per component.
// The RK update (Iteration*), the CFS-PML auxiliaries and the free-surface
// work (VLOW operators, surface matrices, traction image) are fused into the
// same pass; there are no derivative or hW arrays.
//
// Per cell the arithmetic is that of the reference's CalDiffmix + CalWavemix
// + CalTIMGmix + Iteration* (src/calculate.cu:4121-4621, 5668-5897,
// 6330-6734); point sources are added by a separate tiny kernel (solver.cu).
//
// Every wait on an mbarrier is bounded (about 2 s of %globaltimer).  On
// expiry the CTA leaves the march together (the flag is read after a
// barrier), records an error code in *err, waits (bounded) for its own copies
// still in flight and returns; the host then reports CGFD_ERR_TIMEOUT.  Before
// issuing any copy the CTA checks the alignment of its slots and barriers.
#pragma once

#include "cgfd_internal.cuh"
#include "ptx_util.cuh"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <new>

namespace cgfd {
namespace fused {
using namespace ptx;

constexpr int TX = 32, TY = 4, TT = TX * TY;   // threads per CTA tile
constexpr int BOXX = TX + 8, BOXY = TY + 6;    // halo box (x starts 4 left, y 3 below)
constexpr int NSLOT = 5;
constexpr int PLANE = BOXX * BOXY;             // floats per component per halo plane
enum { PART_VEL = 0, PART_STR = 1 };

// NC: staged (differentiated) components, C0: first of them in a set;
// NS: components the part updates (V: 3, T: 6), S0 their first index;
// NCOEF: media coefficients it reads, COEF0 the first (lam2mu, mu, irho).
template <int PART> struct PartInfo;
template <> struct PartInfo<PART_VEL> {
  static constexpr int NC = 6, C0 = TXX, NS = 3, S0 = VX, NCOEF = 1, COEF0 = 2;
};
template <> struct PartInfo<PART_STR> {
  static constexpr int NC = 3, C0 = VX, NS = 6, S0 = TXX, NCOEF = 2, COEF0 = 0;
};

// Slot layout (floats): halo [NC][BOXY][BOXX], then pointwise tiles of TT
// floats: u0 [NS] (FW, or tW in the final stage), u1 [NS] (tW in the inner
// stages), coef [NCOEF], met [3] (zeta_x, zeta_y, zeta_z).  A tensor copy
// needs a 128-byte aligned shared-memory destination: every region starts on
// 128 B (TT floats = 512 B) and the slot stride is a multiple of 128 B.
template <int PART> struct Slot {
  static constexpr int NC = PartInfo<PART>::NC, NS = PartInfo<PART>::NS;
  static constexpr uint32_t HALO_B = (uint32_t)(PLANE * NC * 4);
  static constexpr uint32_t HALO_F = (HALO_B + 127u) / 128u * 32u;  // floats, padded
  static constexpr uint32_t U0 = HALO_F, U1 = U0 + NS * TT, COEF = U1 + NS * TT;
  static constexpr uint32_t MET = COEF + PartInfo<PART>::NCOEF * TT;
  static constexpr uint32_t FLOATS = MET + 3 * TT;
  static constexpr uint32_t BYTES = FLOATS * 4;
  static constexpr size_t SMEM = (size_t)NSLOT * BYTES + 128 + 128;  // + barriers, align slack
};
static_assert(Slot<PART_VEL>::BYTES % 128 == 0 && Slot<PART_STR>::BYTES % 128 == 0, "slots");
static_assert((Slot<PART_VEL>::U0 * 4) % 128 == 0 && (Slot<PART_STR>::U0 * 4) % 128 == 0, "u0");

// Tensor maps of one stage launch.
struct StageMaps {
  CUtensorMap halo;  // stage input, box {40, 10, 1, NC}
  CUtensorMap u0;    // FW (or tW), box {32, 4, 1, NS}
  CUtensorMap u1;    // tW, box {32, 4, 1, NS}
  CUtensorMap coef;  // media, box {32, 4, 1, NCOEF}
  CUtensorMap met;   // metric, box {32, 4, 1, 3}
};

__device__ __forceinline__ float drp5(float m1, float c0, float p1, float p2, float p3, float r) {
  return (CGFD_DA_1 * m1 + CGFD_DA0 * c0 + CGFD_DA1 * p1 + CGFD_DA2 * p2 + CGFD_DA3 * p3) * r;
}

// RK update of one value (Iteration*): KIND 0 first stage (u0 = FW),
// 1 inner (u0 = FW, u1 = tW), 2 final (u0 = tW)
template <int KIND>
__device__ __forceinline__ void rk_store(float *out, float *tw, size_t o, float u0, float u1,
                                         float hh, float adt, float bdt) {
  if (KIND == 0) {
    out[o] = u0 + adt * hh;
    tw[o] = u0 + bdt * hh;
  } else if (KIND == 1) {
    out[o] = u0 + adt * hh;
    tw[o] = u1 + bdt * hh;
  } else {
    out[o] = u0 + bdt * hh;
  }
}
// ADE auxiliaries of one cell and direction: every load first (all in flight
// together, issued before the stencil arithmetic), the stores at the end.
// ai = stage input (FA in the first stage, A after), af = FA, at = tA.
template <int KIND, int N>
struct Aux {
  float ai[N], af[N], at[N];
  __device__ __forceinline__ void load(const StageArgs &a, int d, size_t p, int c0) {
    const size_t as = a.g.astride[d];
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const size_t o = (c0 + q) * as + p;
      ai[q] = a.ain[d][o];
    }
  }
  // RK operands (FA, tA), loaded together right before the stores
  __device__ __forceinline__ void load_rk(const StageArgs &a, int d, size_t p, int c0) {
    const size_t as = a.g.astride[d];
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const size_t o = (c0 + q) * as + p;
      if (KIND == 1) af[q] = a.afw[d][o];
      if (KIND != 0) at[q] = a.ta[d][o];
    }
  }
  __device__ __forceinline__ void store(const StageArgs &a, int d, size_t p, int c0,
                                        const float *hh) const {
    const size_t as = a.g.astride[d];
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const size_t o = (c0 + q) * as + p;
      if (KIND == 0) {
        a.aout[d][o] = ai[q] + a.adt * hh[q];
        a.ta[d][o] = ai[q] + a.bdt * hh[q];
      } else if (KIND == 1) {
        a.aout[d][o] = af[q] + a.adt * hh[q];
        a.ta[d][o] = at[q] + a.bdt * hh[q];
      } else {
        a.aout[d][o] = at[q] + a.bdt * hh[q];
      }
    }
  }
};

// Per-cell context shared by the two parts.
struct Cell {
  int i, j, k, ix, iy, iz;
  int xa, ya;        // compact aux x / y index of the column
  size_t c;          // linear index
  bool top, near_top, zpml, xpml, ypml, interior;
  float iBx, iBy;
};

// boundary-path quantities of a cell, computed only where they are needed
struct Edge {
  float iBz;
  size_t px, py, pz;  // aux indices
  __device__ Edge() : iBz(1.f), px(0), py(0), pz(0) {}
  __device__ Edge(const StageArgs &a, const Cell &e) {
    const Geom &g = a.g;
    iBz = 1.f / a.b[2][e.iz];
    px = ((size_t)e.iz * g.nyi + e.iy) * g.nxa + e.xa;
    py = ((size_t)e.iz * g.nya + e.ya) * g.px + e.ix;
    const int za = (e.k < g.nabs[4]) ? e.k : e.k - (g.nk - g.nabs[5]) + g.nabs[4];
    pz = ((size_t)za * g.nyi + e.iy) * g.px + e.ix;
  }
};

// Pointwise operands of the current plane in shared memory.
struct Pw {
  const float *u0, *u1, *coef, *met;  // already offset to this thread's column
  __device__ float U0(int q) const { return u0[q * TT]; }
  __device__ float U1(int q) const { return u1[q * TT]; }
  __device__ float C(int q) const { return coef[q * TT]; }
  __device__ float M(int q) const { return met[q * TT]; }
};

// -------------------------- velocity part ---------------------------------
// dV/dt = (1/rho) (d_xi sigma_x + d_eta sigma_y + zeta . d_zeta sigma), each
// directional part divided by its CFS beta; ADE auxiliaries for V.  The top 3
// layers take the traction image instead (timg.cu).
template <int X, int Y, int Z, int KIND, int LAG>
__device__ __forceinline__ void vel_cell(const StageArgs &a, const Cell &e, const float *P,
                                         int sc, const Pw &pw, const float (&w)[6][5],
                                         float rx, float ry, float rz) {
  const Geom &g = a.g;
  const size_t fs = g.fstride;
  // staged components: 0 Txx 1 Tyy 2 Tzz 3 Txy 4 Txz 5 Tyz
  auto xs = [&](int s, int d) { return P[s * PLANE + sc + X * d]; };
  auto ys = [&](int s, int d) { return P[s * PLANE + sc + Y * d * BOXX]; };
  auto zs = [&](int s, int d) { return w[s][LAG + Z * d]; };
  auto dx = [&](int s) { return drp5(xs(s, -1), xs(s, 0), xs(s, 1), xs(s, 2), xs(s, 3), rx); };
  auto dy = [&](int s) { return drp5(ys(s, -1), ys(s, 0), ys(s, 1), ys(s, 2), ys(s, 3), ry); };
  auto dz = [&](int s) { return drp5(zs(s, -1), zs(s, 0), zs(s, 1), zs(s, 2), zs(s, 3), rz); };

  // boundary cells: issue every auxiliary load before the stencil arithmetic
  const bool bnd = !e.interior;
  Edge ed;
  Aux<KIND, 3> ax, ay, az;
  if (bnd) {
    ed = Edge(a, e);
    if (e.xpml) ax.load(a, 0, ed.px, 0);
    if (e.ypml) ay.load(a, 1, ed.py, 0);
    if (e.zpml) az.load(a, 2, ed.pz, 0);
  }
  const float irho = pw.C(0);
  float ztx = 0.f, zty = 0.f, ztz = 1.f;
  const bool curved = e.iz >= g.con && !a.flat;
  if (!a.flat) {
    ztz = pw.M(2);
    if (curved) { ztx = pw.M(0); zty = pw.M(1); }
  }
  float dxi[3], det[3], dzt[3];
  dxi[0] = dx(0) * irho;  // DxTxx
  dxi[1] = dx(3) * irho;  // DxTxy
  dxi[2] = dx(4) * irho;  // DxTxz
  det[0] = dy(3) * irho;  // DyTxy
  det[1] = dy(1) * irho;  // DyTyy
  det[2] = dy(5) * irho;  // DyTyz
  const float DzTzz = dz(2), DzTxz = dz(4), DzTyz = dz(5);
  if (curved) {
    const float DzTxx = dz(0), DzTyy = dz(1), DzTxy = dz(3);
    dzt[0] = (ztx * DzTxx + zty * DzTxy + ztz * DzTxz) * irho;
    dzt[1] = (ztx * DzTxy + zty * DzTyy + ztz * DzTyz) * irho;
    dzt[2] = (ztx * DzTxz + zty * DzTyz + ztz * DzTzz) * irho;
  } else {
    dzt[0] = ztz * DzTxz * irho;
    dzt[1] = ztz * DzTyz * irho;
    dzt[2] = ztz * DzTzz * irho;
  }
  float hw[3];
  if (e.interior) {
#pragma unroll
    for (int q = 0; q < 3; ++q) hw[q] = dxi[q] + det[q] + dzt[q];
  } else {
#pragma unroll
    for (int q = 0; q < 3; ++q) hw[q] = dxi[q] * e.iBx + det[q] * e.iBy + dzt[q] * ed.iBz;
    float hax[3], hay[3], haz[3];
    if (e.xpml) {
      const float APD = a.apd[0][e.ix], DB = a.db[0][e.ix];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        hw[q] -= ax.ai[q] * e.iBx;
        hax[q] = dxi[q] * DB - APD * ax.ai[q];
      }
    }
    if (e.ypml) {
      const float APD = a.apd[1][e.iy], DB = a.db[1][e.iy];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        hw[q] -= ay.ai[q] * e.iBy;
        hay[q] = det[q] * DB - APD * ay.ai[q];
      }
    }
    if (e.zpml) {
      const float APD = a.apd[2][e.iz], DB = a.db[2][e.iz];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        hw[q] -= az.ai[q] * ed.iBz;
        haz[q] = dzt[q] * DB - APD * az.ai[q];
      }
    }
    // the top 3 layers' velocities (and their x/y auxiliaries) come from the
    // traction-image kernel (timg.cu); only the z auxiliaries are kept here
    const bool xy = !e.near_top;
    if (e.xpml && xy) ax.load_rk(a, 0, ed.px, 0);
    if (e.ypml && xy) ay.load_rk(a, 1, ed.py, 0);
    if (e.zpml) az.load_rk(a, 2, ed.pz, 0);
    if (e.xpml && xy) ax.store(a, 0, ed.px, 0, hax);
    if (e.ypml && xy) ay.store(a, 1, ed.py, 0, hay);
    if (e.zpml) az.store(a, 2, ed.pz, 0, haz);
    if (!xy) return;
  }
#pragma unroll
  for (int q = 0; q < 3; ++q)
    rk_store<KIND>(static_cast<float *>(a.out), static_cast<float *>(a.tw), (size_t)(VX + q) * fs + e.c, pw.U0(q),
                   KIND == 1 ? pw.U1(q) : 0.f, hw[q], a.adt, a.bdt);
}

// --------------------------- stress part ----------------------------------
// dsigma/dt from Hooke's law with the velocity gradient in curvilinear form;
// the surface-layer d/dzeta of V comes from the traction-free matrices, the
// next two layers use the 2-point and Gottlieb 2-4 operators (VLOW).
template <int X, int Y, int Z, int KIND, int LAG>
__device__ __forceinline__ void str_cell(const StageArgs &a, const Cell &e, const float *P,
                                         int sc, const Pw &pw, const float (&w)[3][5],
                                         float rx, float ry, float rz) {
  const Geom &g = a.g;
  const size_t fs = g.fstride;
  auto xs = [&](int s, int d) { return P[s * PLANE + sc + X * d]; };
  auto ys = [&](int s, int d) { return P[s * PLANE + sc + Y * d * BOXX]; };
  auto zs = [&](int s, int d) { return w[s][LAG + Z * d]; };
  auto dx = [&](int s) { return drp5(xs(s, -1), xs(s, 0), xs(s, 1), xs(s, 2), xs(s, 3), rx); };
  auto dy = [&](int s) { return drp5(ys(s, -1), ys(s, 0), ys(s, 1), ys(s, 2), ys(s, 3), ry); };
  auto dz = [&](int s) { return drp5(zs(s, -1), zs(s, 0), zs(s, 1), zs(s, 2), zs(s, 3), rz); };

  // boundary cells: issue every auxiliary load before the stencil arithmetic
  const bool bnd = !e.interior;
  Edge ed;
  Aux<KIND, 6> ax, ay, az;
  if (bnd) {
    ed = Edge(a, e);
    if (e.xpml) ax.load(a, 0, ed.px, 3);
    if (e.ypml) ay.load(a, 1, ed.py, 3);
    if (e.zpml) az.load(a, 2, ed.pz, 3);
  }
  const float DxVx = dx(0), DxVy = dx(1), DxVz = dx(2);
  const float DyVx = dy(0), DyVy = dy(1), DyVz = dy(2);
  float DzVx, DzVy, DzVz;
  float cx[9], cy[9];
  if (e.top) {
    const size_t m2 = (size_t)e.iy * g.px + e.ix;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      cx[q] = a.matv[q * g.plane + m2];
      cy[q] = a.matv[(9 + q) * g.plane + m2];
    }
    DzVx = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz + cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz;
    DzVy = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz + cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz;
    DzVz = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz + cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz;
  } else if (e.iz == g.top - 1) {  // 2-point (M22)
    DzVx = (zs(0, 1) - zs(0, 0)) * rz;
    DzVy = (zs(1, 1) - zs(1, 0)) * rz;
    DzVz = (zs(2, 1) - zs(2, 0)) * rz;
  } else if (e.iz == g.top - 2) {  // Gottlieb 2-4 (M24)
    DzVx = (CGFD_MA0 * zs(0, 0) + CGFD_MA1 * zs(0, 1) + CGFD_MA2 * zs(0, 2)) * rz;
    DzVy = (CGFD_MA0 * zs(1, 0) + CGFD_MA1 * zs(1, 1) + CGFD_MA2 * zs(1, 2)) * rz;
    DzVz = (CGFD_MA0 * zs(2, 0) + CGFD_MA1 * zs(2, 1) + CGFD_MA2 * zs(2, 2)) * rz;
  } else {
    DzVx = dz(0); DzVy = dz(1); DzVz = dz(2);
  }

  const float lam2mu = pw.C(0), miu = pw.C(1);
  const float lambda = lam2mu - 2.f * miu;
  float ztx = 0.f, zty = 0.f, ztz = 1.f;
  if (!a.flat) {
    ztz = pw.M(2);
    if (e.iz >= g.con) { ztx = pw.M(0); zty = pw.M(1); }
  }
  // components in the set order Txx Tyy Tzz Txy Txz Tyz (index q = comp - 3)
  float dxi[6], det[6], dzt[6];
  dxi[0] = lam2mu * DxVx; det[0] = lambda * DyVy;
  dzt[0] = lam2mu * ztx * DzVx + lambda * zty * DzVy + lambda * ztz * DzVz;
  dxi[1] = lambda * DxVx; det[1] = lam2mu * DyVy;
  dzt[1] = lambda * ztx * DzVx + lam2mu * zty * DzVy + lambda * ztz * DzVz;
  dxi[2] = lambda * DxVx; det[2] = lambda * DyVy;
  dzt[2] = lambda * ztx * DzVx + lambda * zty * DzVy + lam2mu * ztz * DzVz;
  dxi[3] = DxVy * miu; det[3] = DyVx * miu; dzt[3] = (zty * DzVx + ztx * DzVy) * miu;
  dxi[4] = DxVz * miu; det[4] = 0.f;        dzt[4] = (ztz * DzVx + ztx * DzVz) * miu;
  dxi[5] = 0.f;        det[5] = DyVz * miu; dzt[5] = (ztz * DzVy + zty * DzVz) * miu;

  float hw[6];
  if (e.interior) {
#pragma unroll
    for (int q = 0; q < 6; ++q) hw[q] = dxi[q] + det[q] + dzt[q];
  } else {
#pragma unroll
    for (int q = 0; q < 6; ++q) hw[q] = dxi[q] * e.iBx + det[q] * e.iBy + dzt[q] * ed.iBz;
    float hax[6], hay[6], haz[6];
    // surface layer: the ADE auxiliaries also take the xi (eta) part of the
    // surface-matrix d/dzeta of V (src/calculate.cu:4479-4491, 4527-4538)
    auto surf = [&](float z1v, float z2v, float z3v, float f, float *out) {
      out[0] += f * (lam2mu * ztx * z1v + lambda * zty * z2v + lambda * ztz * z3v);
      out[1] += f * (lambda * ztx * z1v + lam2mu * zty * z2v + lambda * ztz * z3v);
      out[2] += f * (lambda * ztx * z1v + lambda * zty * z2v + lam2mu * ztz * z3v);
      out[3] += f * (zty * z1v + ztx * z2v) * miu;
      out[4] += f * (ztz * z1v + ztx * z3v) * miu;
      out[5] += f * (ztz * z2v + zty * z3v) * miu;
    };
    if (e.xpml) {
      const float APD = a.apd[0][e.ix], DB = a.db[0][e.ix];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        hw[q] -= ax.ai[q] * e.iBx;
        hax[q] = dxi[q] * DB - APD * ax.ai[q];
      }
      if (e.top)
        surf(cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz, cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz,
             cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz, DB * a.b[0][e.ix], hax);
    }
    if (e.ypml) {
      const float APD = a.apd[1][e.iy], DB = a.db[1][e.iy];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        hw[q] -= ay.ai[q] * e.iBy;
        hay[q] = det[q] * DB - APD * ay.ai[q];
      }
      if (e.top)
        surf(cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz, cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz,
             cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz, DB * a.b[1][e.iy], hay);
    }
    if (e.zpml) {
      const float APD = a.apd[2][e.iz], DB = a.db[2][e.iz];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        hw[q] -= az.ai[q] * ed.iBz;
        haz[q] = dzt[q] * DB - APD * az.ai[q];
      }
    }
    if (e.xpml) ax.load_rk(a, 0, ed.px, 3);
    if (e.ypml) ay.load_rk(a, 1, ed.py, 3);
    if (e.zpml) az.load_rk(a, 2, ed.pz, 3);
    if (e.xpml) ax.store(a, 0, ed.px, 3, hax);
    if (e.ypml) ay.store(a, 1, ed.py, 3, hay);
    if (e.zpml) az.store(a, 2, ed.pz, 3, haz);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q)
    rk_store<KIND>(static_cast<float *>(a.out), static_cast<float *>(a.tw), (size_t)(TXX + q) * fs + e.c, pw.U0(q),
                   KIND == 1 ? pw.U1(q) : 0.f, hw[q], a.adt, a.bdt);
}

// ------------------------------ the march ---------------------------------
// items: tile index fastest, so the CTAs resident at one time work on
// neighbouring tiles of the same z-chunk and share halo rows in L2
template <int PART, int X, int Y, int Z, int KIND>
__global__ void __launch_bounds__(TT, 3)
    stage_part_kernel(const __grid_constant__ StageMaps maps, const StageArgs a, int zchunk,
                      int ntx, int ntiles, int nitems, int *err) {
  using S = Slot<PART>;
  constexpr int NC = PartInfo<PART>::NC, C0 = PartInfo<PART>::C0;
  constexpr int NS = PartInfo<PART>::NS, S0 = PartInfo<PART>::S0;
  constexpr int NCOEF = PartInfo<PART>::NCOEF, COEF0 = PartInfo<PART>::COEF0;
  constexpr int LEAD = (Z > 0) ? 3 : 1, LAG = (Z > 0) ? 1 : 3;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // align the ring on the shared-window address itself
  unsigned char *base = smem_raw + ((128u - (su32(smem_raw) & 127u)) & 127u);
  float *ring = reinterpret_cast<float *>(base);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + (size_t)NSLOT * S::BYTES);
  __shared__ int abort_flag;

  const Geom &g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const size_t fs = g.fstride;
  const bool flat = a.flat;
  // bytes one plane delivers: halo always, pointwise only for computed planes
  const uint32_t pw_bytes = (uint32_t)(TT * 4) *
      (NS * (KIND == 1 ? 2 : 1) + NCOEF + (flat ? 0 : 3));

  if (tid == 0) {
    abort_flag = 0;
    bool aligned = ((su32(bars) & 7u) == 0);
    for (int s = 0; s < NSLOT; ++s)
      aligned = aligned && ((su32(ring + (size_t)s * S::FLOATS) & 127u) == 0);
    if (!aligned) {
      abort_flag = 1;
      if (err) atomicExch(err, 2);
    } else {
      for (int s = 0; s < NSLOT; ++s) mbar_init(&bars[s], 1);
      fence_mbar_init();
    }
  }
  __syncthreads();
  if (abort_flag) return;  // nothing was issued

  uint32_t ph = 0;    // parity of the next wait, per slot (same in every thread)
  uint32_t pend = 0;  // thread 0: slots with a copy not yet waited for
  const float rx = (float)X / a.h, ry = (float)Y / a.h, rz = (float)Z / a.h;
  const int sc = (ty + 3) * BOXX + (tx + 4);  // this column inside a halo plane

  for (int item = blockIdx.x; item < nitems && !abort_flag; item += gridDim.x) {
    const int tile = item % ntiles, cz = item / ntiles;
    const int bx0 = (tile % ntx) * TX, by0 = (tile / ntx) * TY;
    const int z0 = LFD + cz * zchunk;
    const int z1 = min(z0 + zchunk, g.nk + LFD);
    const int pmax = z1 - 1 + LEAD;  // last plane the chunk reads
    auto issue = [&](int p) {        // thread 0 only
      const int s = (p - z0) % NSLOT;
      float *slot = ring + (size_t)s * S::FLOATS;
      const bool compute = p < z1;
      fence_proxy_async();
      mbar_expect_tx(&bars[s], S::HALO_B + (compute ? pw_bytes : 0u));
      tma_load(slot, &maps.halo, bx0 + XO - 4, by0, p, C0, &bars[s]);
      if (compute) {
        const int cx = XO + bx0, cy = LFD + by0;
        tma_load(slot + S::U0, &maps.u0, cx, cy, p, S0, &bars[s]);
        if (KIND == 1) tma_load(slot + S::U1, &maps.u1, cx, cy, p, S0, &bars[s]);
        tma_load(slot + S::COEF, &maps.coef, cx, cy, p, COEF0, &bars[s]);
        if (!flat) tma_load(slot + S::MET, &maps.met, cx, cy, p, 0, &bars[s]);
      }
      pend |= 1u << s;
    };
    auto wait = [&](int p) -> bool {  // every thread, in plane order
      const int s = (p - z0) % NSLOT;
      const bool ok = mbar_wait(&bars[s], (ph >> s) & 1u);
      if (ok) {  // an expired wait leaves the copy pending for the drain
        ph ^= 1u << s;
        if (tid == 0) pend &= ~(1u << s);
      }
      return ok;
    };
    if (tid == 0)
      for (int p = z0; p < z0 + NSLOT && p <= pmax; ++p) issue(p);

    Cell e;
    e.i = bx0 + tx;
    e.j = by0 + ty;
    const bool active = (e.i < g.ni) && (e.j < g.nj);
    e.ix = e.i + XO;
    e.iy = e.j + LFD;
    e.xpml = active && (e.i < g.nabs[0] || e.i >= g.ni - g.nabs[1]);
    e.ypml = active && (e.j < g.nabs[2] || e.j >= g.nj - g.nabs[3]);
    e.xa = (e.i < g.nabs[0]) ? e.i : e.i - (g.ni - g.nabs[1]) + g.xaoff;
    e.ya = (e.j < g.nabs[2]) ? e.j : e.j - (g.nj - g.nabs[3]) + g.nabs[2];
    e.iBx = 1.f / a.b[0][e.ix];
    e.iBy = 1.f / a.b[1][e.iy];
    // tile-uniform: no x/y PML anywhere in this tile (and B = 1, DB = APD = 0
    // outside the layers, which the solver checks at upload)
    const bool tile_xy_interior =
        a.plain_interior && (bx0 >= g.nabs[0]) && (bx0 + TX <= g.ni - g.nabs[1]) &&
        (by0 >= g.nabs[2]) && (by0 + TY <= g.nj - g.nabs[3]);

    // register windows: w[c][0..4] = planes iz-LAG .. iz+LEAD at this column
    float w[NC][5];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int q = 0; q < 5; ++q) w[c][q] = 0.f;
    auto push = [&](const float *src, size_t stride, size_t off) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
#pragma unroll
        for (int q = 0; q < 4; ++q) w[c][q] = w[c][q + 1];
        w[c][4] = src[c * stride + off];
      }
    };
    // planes below the chunk come straight from global memory (centre only)
    for (int p = z0 - LAG; p < z0; ++p) {
      if (active) push(static_cast<const float *>(a.in) + (size_t)C0 * fs, fs, gidx(g, e.ix, e.iy, p));
      else push(ring, 0, 0);  // keeps the window shape; values unused
    }
    // A wait that expires sets the CTA-wide abort flag; the flag is read only
    // after a __syncthreads, so every thread leaves the march together.
    for (int p = z0; p < z0 + LEAD; ++p) {
      if (wait(p)) push(ring + (size_t)((p - z0) % NSLOT) * S::FLOATS, PLANE, sc);
      else abort_flag = 1;
    }
    __syncthreads();

    // plane iz lives in slot (iz - z0) % NSLOT
    const int tc = ty * TX + tx;
    const int zlo = LFD + g.nabs[4], zhi = g.nk + LFD - g.nabs[5];  // z interior [zlo, zhi)
    size_t cidx = gidx(g, e.ix, e.iy, z0);
    int slot_c = 0, slot_n = LEAD % NSLOT;  // slots of plane iz and of plane iz+LEAD
    for (int iz = z0; iz < z1; ++iz) {
      const bool got = wait(iz + LEAD);
      if (got) push(ring + (size_t)slot_n * S::FLOATS, PLANE, sc);
      else abort_flag = 1;
      if (active && got) {
        const float *slot = ring + (size_t)slot_c * S::FLOATS;
        Pw pw{slot + S::U0 + tc, slot + S::U1 + tc, slot + S::COEF + tc, slot + S::MET + tc};
        e.iz = iz;
        e.k = iz - LFD;
        e.c = cidx;
        e.top = (iz == g.top);
        e.near_top = iz >= g.top - 2;
        e.zpml = (iz < zlo) || (iz >= zhi);
        e.interior = tile_xy_interior && !e.zpml && !e.near_top;
        if constexpr (PART == PART_VEL)
          vel_cell<X, Y, Z, KIND, LAG>(a, e, slot, sc, pw, w, rx, ry, rz);
        else
          str_cell<X, Y, Z, KIND, LAG>(a, e, slot, sc, pw, w, rx, ry, rz);
      }
      // the slot of plane iz is free: refill it with plane iz+NSLOT
      __syncthreads();
      if (abort_flag) break;
      if (tid == 0 && iz + NSLOT <= pmax) issue(iz + NSLOT);
      cidx += g.plane;
      slot_c = (slot_c + 1 == NSLOT) ? 0 : slot_c + 1;
      slot_n = (slot_n + 1 == NSLOT) ? 0 : slot_n + 1;
    }
    __syncthreads();  // all reads of the ring done before the next item reuses it
  }
  if (abort_flag && tid == 0) {
    if (err) atomicExch(err, 1);
    // drain: wait (bounded) for copies still in flight before the CTA's
    // shared memory goes away
    for (int s = 0; s < NSLOT; ++s)
      if (pend & (1u << s)) mbar_wait(&bars[s], (ph >> s) & 1u);
  }
}

struct Plan {
  // per field set (FW, Wa, Wb, tW): halo boxes for the two parts and the
  // pointwise boxes of V (3) and T (6) components
  CUtensorMap haloV[4], haloS[4], ctrV[4], ctrT[4];
  CUtensorMap coefV, coefS, met;
  int zchunk, ntx, ntiles, nitems, grid[2];
};

template <int PART, int X, int Y, int Z, int KIND>
void launch_t(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err, cudaStream_t s) {
  stage_part_kernel<PART, X, Y, Z, KIND><<<pl.grid[PART], dim3(TX, TY, 1), Slot<PART>::SMEM, s>>>(
      m, a, pl.zchunk, pl.ntx, pl.ntiles, pl.nitems, err);
}

template <int PART, int KIND>
void launch_dirs(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err,
                 cudaStream_t s) {
  const int code = (a.X > 0 ? 4 : 0) + (a.Y > 0 ? 2 : 0) + (a.Z > 0 ? 1 : 0);
  switch (code) {
    case 0: launch_t<PART, -1, -1, -1, KIND>(pl, m, a, err, s); break;
    case 1: launch_t<PART, -1, -1, 1, KIND>(pl, m, a, err, s); break;
    case 2: launch_t<PART, -1, 1, -1, KIND>(pl, m, a, err, s); break;
    case 3: launch_t<PART, -1, 1, 1, KIND>(pl, m, a, err, s); break;
    case 4: launch_t<PART, 1, -1, -1, KIND>(pl, m, a, err, s); break;
    case 5: launch_t<PART, 1, -1, 1, KIND>(pl, m, a, err, s); break;
    case 6: launch_t<PART, 1, 1, -1, KIND>(pl, m, a, err, s); break;
    default: launch_t<PART, 1, 1, 1, KIND>(pl, m, a, err, s); break;
  }
}

template <int PART, int KIND>
void set_attrs() {
  auto set = [](const void *f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Slot<PART>::SMEM);
  };
  set((const void *)stage_part_kernel<PART, -1, -1, -1, KIND>);
  set((const void *)stage_part_kernel<PART, -1, -1, 1, KIND>);
  set((const void *)stage_part_kernel<PART, -1, 1, -1, KIND>);
  set((const void *)stage_part_kernel<PART, -1, 1, 1, KIND>);
  set((const void *)stage_part_kernel<PART, 1, -1, -1, KIND>);
  set((const void *)stage_part_kernel<PART, 1, -1, 1, KIND>);
  set((const void *)stage_part_kernel<PART, 1, 1, -1, KIND>);
  set((const void *)stage_part_kernel<PART, 1, 1, 1, KIND>);
}

template <int PART>
int resident_ctas() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per, stage_part_kernel<PART, 1, 1, 1, 1>, TT, Slot<PART>::SMEM);
  if (per < 1) per = 1;
  if (sms < 1) sms = 1;
  return per * sms;
}

// per-(part, kind) entry points, one translation unit each (fused_*.cu)
#define CGFD_FUSED_DECL(P, K)                                                        \
  void launch_##P##K(const Plan &pl, const StageMaps &m, const StageArgs &a, int *err, \
                     cudaStream_t s);                                                \
  void attrs_##P##K();
CGFD_FUSED_DECL(v, 0)
CGFD_FUSED_DECL(v, 1)
CGFD_FUSED_DECL(v, 2)
CGFD_FUSED_DECL(s, 0)
CGFD_FUSED_DECL(s, 1)
CGFD_FUSED_DECL(s, 2)
#undef CGFD_FUSED_DECL
int resident_vel();
int resident_str();

}  // namespace fused
}  // namespace cgfd
