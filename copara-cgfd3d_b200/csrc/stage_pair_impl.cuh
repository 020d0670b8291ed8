// stage_pair_impl.cuh -- z-marching RK stage kernels for sm_100a with two
// x-adjacent cells per thread (templates; instantiated by pair_*.cu).
//
// One RK stage is two kernels, split along the velocity-stress structure of
// the equations: the velocity part differentiates only the six stresses and
// the stress part only the three velocities.  A CTA of 32 x 4 threads owns a
// tile of 64 x 4 (x, y) columns, each thread the cell pair (2t, 2t+1) of its
// row, and marches through a chunk of z-planes; a persistent grid of CTAs
// (two per SM) walks the (tile, z-chunk) items.
//
// Pairs make every per-cell quantity a float2: the stencil and RHS
// arithmetic runs as packed FFMA2 / FMUL2 / FADD2 (one instruction for both
// cells), and the shared-memory reads, the pointwise operands and the
// global stores are 64-bit accesses.  Only the x-derivative assembles some of
// its operand pairs from neighbouring pairs.
//
// The march runs against the long reach of the z-stencil: a forward stencil
// (reach -1..+3) marches downwards, a backward one (reach -3..+1) upwards, so
// the stencil always needs one plane ahead and three behind.  Each plane
// arrives by TMA (cp.async.bulk.tensor, no multicast) into one slot of a
// 4-slot shared-memory ring, on one mbarrier per slot:
//   * the differentiated components with an x/y halo, one 4-D box
//     {72 x, 10 y, 1 z, NC components} (x from -4, y from -3);
//   * the pointwise operands of the plane, boxes {64, 4, 1, n}: the RK
//     registers (FW and/or tW), the media coefficients and the metric.
// A plane is needed one iteration after it lands (its centre enters the
// per-thread register window of five planes) and in the next one (x/y
// stencils, pointwise operands); two further planes are in flight.
//
// The per-cell arithmetic is that of the reference's CalDiffmix + CalWavemix
// + Iteration* (src/calculate.cu:4121-4621, 6330-6734); the top three layers'
// velocities come from the traction-image kernel (timg.cu) and point sources
// from a separate tiny kernel (solver.cu).  CFS-PML auxiliaries are read and
// written with 64-bit global accesses (prefetched into L2 by tensor prefetch
// when the plane's slot is issued).
//
// Every mbarrier wait is bounded (about 2 s of %globaltimer).  On expiry the
// CTA leaves the march together (the flag is read after a barrier), records
// an error code in *err, waits (bounded) for its own copies still in flight
// and returns; the host then reports CGFD_ERR_TIMEOUT.  Before issuing any
// copy the CTA checks the alignment of its slots and barriers (error code 2).
#pragma once

#include "cgfd_internal.cuh"
#include "ptx_util.cuh"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <vector>

namespace cgfd {
namespace pair {
using namespace ptx;

constexpr int TX = 32, TY = 4, TT = TX * TY;  // threads per CTA
constexpr int CX = 2 * TX;                    // cells per tile row
constexpr int HY = TY + 6;                    // halo box rows (y from -3)
constexpr int PWT = CX * TY;                  // values per pointwise tile
// halo box columns per storage type: x from -HOFF, so that the box origin is
// 16-byte aligned (x from -4 for FP32, -8 for 16-bit storage)
template <typename T> struct Halo {
  static constexpr int HOFF = (sizeof(T) == 4) ? 4 : 8;
  static constexpr int HX = CX + 2 * HOFF;
  static constexpr int HPL = HX * HY;  // values per component per halo plane
};
constexpr int NSLOT = 4;
enum { PART_VEL = 0, PART_STR = 1 };
#ifndef CGFD_PAIR_UNROLL
#define CGFD_PAIR_UNROLL 1
#endif
constexpr int MARCH_UNROLL = CGFD_PAIR_UNROLL;  // unroll factor of the march loop

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

// Slot layout (byte offsets): halo [NC][HY][HX] of the storage type T, then
// pointwise tiles of PWT values: u0 [NS] (FW, or tW in the final stage) and
// u1 [NS] (tW in the inner stages) of type T, coef [NCOEF] and met [3]
// (zeta_x, zeta_y, zeta_z) of FP32.  Every region starts on 128 B (a tensor
// copy's shared-memory destination must) and the slot stride is a multiple
// of 128 B.
constexpr uint32_t up128(uint32_t b) { return (b + 127u) / 128u * 128u; }
template <typename T, int PART> struct Slot {
  static constexpr int NC = PartInfo<PART>::NC, NS = PartInfo<PART>::NS;
  static constexpr uint32_t HALO_B = (uint32_t)(Halo<T>::HPL * NC * sizeof(T));
  static constexpr uint32_t U0 = up128(HALO_B);
  static constexpr uint32_t U_B = (uint32_t)(NS * PWT * sizeof(T));  // one register set
  static constexpr uint32_t U1 = U0 + up128(U_B);
  static constexpr uint32_t COEF = U1 + up128(U_B);
  static constexpr uint32_t MET = COEF + (uint32_t)(PartInfo<PART>::NCOEF * PWT * 4);
  static constexpr uint32_t BYTES = MET + 3 * PWT * 4;
  static constexpr size_t SMEM = (size_t)NSLOT * BYTES + 128 + 128;  // + barriers, align slack
};
static_assert(Slot<float, PART_VEL>::BYTES % 128 == 0 && Slot<float, PART_STR>::BYTES % 128 == 0,
              "slots");
static_assert(Slot<__half, PART_VEL>::BYTES % 128 == 0 && Slot<__half, PART_STR>::BYTES % 128 == 0,
              "slots");
// two CTAs per SM: 228 KB of shared memory per SM, 1 KB of it reserved per CTA
static_assert(2 * (Slot<float, PART_VEL>::SMEM + 1024) <= 233472, "two velocity CTAs per SM");
static_assert(2 * (Slot<float, PART_STR>::SMEM + 1024) <= 233472, "two stress CTAs per SM");

// resident CTAs per SM the kernels are compiled for.  FP32 storage: two
// (four 27.5 KB slots per CTA; registers <= 255).  16-bit storage: three
// (the slots are about half as large; registers <= 168, a few bytes of
// spills in some instantiations): 6.90 -> 5.79 ms per step on the
// 400x400x200 hill with FP16 storage (with six stress auxiliaries per PML
// direction the stress part needed 248 registers and three CTAs ran slower).
template <typename T> struct MinCtas { static constexpr int value = 2; };
template <> struct MinCtas<__half> { static constexpr int value = 3; };
template <> struct MinCtas<__nv_bfloat16> { static constexpr int value = 3; };
static_assert(3 * (Slot<__half, PART_VEL>::SMEM + 1024) <= 233472, "three 16-bit velocity CTAs");
static_assert(3 * (Slot<__half, PART_STR>::SMEM + 1024) <= 233472, "three 16-bit stress CTAs");

// Tensor maps of one launch.  halo/u0/u1/coef/met feed the ring; the aux
// maps (per direction: stage input, FA, tA) only drive L2 prefetches.
struct Maps {
  CUtensorMap halo;  // stage input, box {72, 10, 1, NC}
  CUtensorMap u0;    // FW (or tW), box {64, 4, 1, NS}
  CUtensorMap u1;    // tW, box {64, 4, 1, NS}
  CUtensorMap coef;  // media, box {64, 4, 1, NCOEF}
  CUtensorMap met;   // metric, box {64, 4, 1, 3}
  CUtensorMap aux[3][3];  // [direction][ain, afw, ta], box {64, 4, 1, NS}
};

// Work list of a launch: items {i0, j0, z0 | z1 << 16, model} (tile
// origin, z range, model of a batch), ordered by decreasing estimated cost;
// CTAs take them in order from an atomic counter (reset before every
// launch), so expensive PML items start first and the cheap interior items
// fill the tail.  A batched launch reads each model's stage arguments and
// tensor maps from the device arrays bargs / bmaps (one entry per model).
struct Work {
  const int4 *items;
  int *counter;       // [0]: velocity launch, [1]: stress launch
  int nitems;
  int has_aux[3];     // direction has a PML (aux maps valid; single model)
  const StageArgs *bargs;
  const Maps *bmaps;
  // bound of every mbarrier wait, and the test hook of cgfd_test_withhold_copy:
  // with withhold >= 0 the velocity part's CTA 0 does not issue the halo copy
  // of entry `withhold` of its first item, so its wait for that plane expires
  unsigned wait_us = WAIT_US;
  int withhold = -1;
};

// ---------------------------- float2 helpers ------------------------------
typedef float2 f2;
__device__ __forceinline__ f2 F2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 S2(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 neg2(f2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ f2 lds2(const float *p) { return *reinterpret_cast<const f2 *>(p); }
// a pair of stored values (any storage type) as float2
template <typename T> __device__ __forceinline__ f2 ldp(const T *p) { return Elem<T>::ld2(p); }
// r times a power-of-two component scale; FP32 storage is unscaled
template <typename T> __device__ __forceinline__ float scaled(float r, float s) {
  if constexpr (sizeof(T) == 4) return r;
  else return r * s;
}

// DRP/opt MacCormack 5-point operator on a pair, in the forward form
// (m1 = p - s, c0 = p, p1..p3 = p + s..3s for the marching sign s; r = s/h)
__device__ __forceinline__ f2 drp2(f2 m1, f2 c0, f2 p1, f2 p2, f2 p3, float r) {
  f2 t = mul2(S2(CGFD_DA_1), m1);
  t = fma2(S2(CGFD_DA0), c0, t);
  t = fma2(S2(CGFD_DA1), p1, t);
  t = fma2(S2(CGFD_DA2), p2, t);
  t = fma2(S2(CGFD_DA3), p3, t);
  return mul2(t, S2(r));
}

// x-derivative of the pair (halo columns cb, cb+1 of row R) with the centre
// pair C already in registers; r = X/h
template <int X, typename T>
__device__ __forceinline__ f2 dx_pair(const T *R, int cb, f2 C, float r) {
  if constexpr (X > 0) {
    const f2 La = ldp(R + cb - 2), Lb = ldp(R + cb + 2), Lc = ldp(R + cb + 4);
    return drp2(F2(La.y, C.x), C, F2(C.y, Lb.x), Lb, F2(Lb.y, Lc.x), r);
  } else {
    const f2 Lz = ldp(R + cb - 4), La = ldp(R + cb - 2), Lb = ldp(R + cb + 2);
    return drp2(F2(C.y, Lb.x), C, F2(La.y, C.x), La, F2(Lz.y, La.x), r);
  }
}
// y-derivative of the pair from the component's halo plane P (row ry of
// this thread, column cb), centre pair C in registers; r = Y/h
template <int Y, typename T>
__device__ __forceinline__ f2 dy_pair(const T *P, int ry, int cb, f2 C, float r) {
  constexpr int HX = Halo<T>::HX;
  const f2 m1 = ldp(P + (ry - Y) * HX + cb), p1 = ldp(P + (ry + Y) * HX + cb);
  const f2 p2 = ldp(P + (ry + 2 * Y) * HX + cb), p3 = ldp(P + (ry + 3 * Y) * HX + cb);
  return drp2(m1, C, p1, p2, p3, r);
}

// masked pair access: bit 0 = first cell, bit 1 = second; p1 is the second
// cell's address (p0 + 1 wherever both bits can be set)
__device__ __forceinline__ f2 ld2(const float *p0, const float *p1, int m) {
  if (m == 3) return *reinterpret_cast<const f2 *>(p0);
  f2 r = F2(0.f, 0.f);
  if (m & 1) r.x = *p0;
  if (m & 2) r.y = *p1;
  return r;
}
__device__ __forceinline__ void st2(float *p0, float *p1, int m, f2 v) {
  if (m == 3) {
    *reinterpret_cast<f2 *>(p0) = v;
  } else {
    if (m & 1) *p0 = v.x;
    if (m & 2) *p1 = v.y;
  }
}
// the same for a field set of storage type T (second cell at p + 1)
template <typename T>
__device__ __forceinline__ f2 ldt2(const T *p, int m) {
  if (m == 3) return Elem<T>::ld2(p);
  f2 r = F2(0.f, 0.f);
  if (m & 1) r.x = Elem<T>::ld(p);
  if (m & 2) r.y = Elem<T>::ld(p + 1);
  return r;
}
template <typename T>
__device__ __forceinline__ void stt2(T *p, int m, f2 v) {
  if (m == 3) {
    Elem<T>::st2(p, v);
  } else {
    if (m & 1) Elem<T>::st(p, v.x);
    if (m & 2) Elem<T>::st(p + 1, v.y);
  }
}

// The per-thread register window of the z-stencil holds the staged
// components as stored: a float2 for FP32, the raw 16-bit pair (one 32-bit
// register) for FP16 / BF16, widened at use.  The widening is exact, so the
// arithmetic is that of a widened window, at half its registers (the 16-bit
// kernels run at 168 registers to fit three CTAs per SM).
template <typename T> struct Win {
  using type = f2;
  __device__ __forceinline__ static f2 get(f2 v) { return v; }
  __device__ __forceinline__ static type ld(const T *p) { return ldp(p); }
  __device__ __forceinline__ static type ldm(const T *p, int m) { return ldt2(p, m); }
  __device__ __forceinline__ static type zero() { return S2(0.f); }
};
template <> struct Win<__half> {
  using type = __half2;
  __device__ __forceinline__ static f2 get(__half2 v) { return __half22float2(v); }
  __device__ __forceinline__ static type ld(const __half *p) {
    return *reinterpret_cast<const __half2 *>(p);
  }
  __device__ __forceinline__ static type zero() { return __float2half2_rn(0.f); }
  __device__ __forceinline__ static type ldm(const __half *p, int m) {
    if (m == 3) return ld(p);
    __half2 r = zero();
    if (m & 1) r.x = p[0];
    if (m & 2) r.y = p[1];
    return r;
  }
};
template <> struct Win<__nv_bfloat16> {
  using type = __nv_bfloat162;
  __device__ __forceinline__ static f2 get(__nv_bfloat162 v) { return __bfloat1622float2(v); }
  __device__ __forceinline__ static type ld(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const __nv_bfloat162 *>(p);
  }
  __device__ __forceinline__ static type zero() { return __float2bfloat162_rn(0.f); }
  __device__ __forceinline__ static type ldm(const __nv_bfloat16 *p, int m) {
    if (m == 3) return ld(p);
    __nv_bfloat162 r = zero();
    if (m & 1) r.x = p[0];
    if (m & 2) r.y = p[1];
    return r;
  }
};

// 16-bit storage keeps the RK accumulator as its difference from the step
// state, tW - FW: the difference is about a time step's change of the field,
// an order of magnitude below the field, so its FP16/BF16 rounding is that
// much finer (the accumulator's rounding was the largest share of the 16-bit
// storage error).  The final stage then reads FW besides it.
template <typename T> struct TwDelta { static constexpr bool value = sizeof(T) != 4; };
// the second pointwise register set is loaded: inner stages (tW, or the stage
// input under tW elision), and the final stage with the difference form (tW)
template <int KIND, typename T> struct TwoRegs {
  static constexpr bool value = KIND == 1 || (KIND == 2 && TwDelta<T>::value);
};

// RK update of one pair (Iteration*): KIND 0 first stage (u0 = FW; no tW
// under tW elision), 1 inner (u0 = FW, u1 = tW; in the second stage under
// elision u1 = the stage input W and tW = FW + rtw*(W - FW) + bdt*h),
// 2 final (u0 = tW; with the difference form u0 = FW and u1 = tW - FW).
// u0, u1 and the outputs are in stored units; adt, bdt carry the component's
// inverse scale (every set of a component shares its scale, so the rebuild
// and the difference are the same in stored units).
template <int KIND, typename T>
__device__ __forceinline__ void rk_store2(const StageArgs &a, T *out, T *tw, int m, f2 u0, f2 u1,
                                          f2 hh, float adt, float bdt) {
  constexpr bool D = TwDelta<T>::value;
  if (KIND == 0) {
    stt2(out, m, fma2(S2(adt), hh, u0));
    if (!a.tw_skip) stt2(tw, m, D ? mul2(S2(bdt), hh) : fma2(S2(bdt), hh, u0));
  } else if (KIND == 1) {
    stt2(out, m, fma2(S2(adt), hh, u0));
    f2 base = u1;
    if (a.tw_skip && a.rk == 1)
      base = D ? mul2(S2(a.rtw), add2(u1, neg2(u0))) : fma2(S2(a.rtw), add2(u1, neg2(u0)), u0);
    stt2(tw, m, fma2(S2(bdt), hh, base));
  } else {
    stt2(out, m, fma2(S2(bdt), hh, D ? add2(u0, u1) : u0));
  }
}

// ADE auxiliaries of one pair and direction: the stage input ai (FA in the
// first stage, A after) enters the RHS and is loaded before the stencil
// arithmetic.  EARLY (FP32 storage, which has the registers): the RK
// registers of the update (FA and tA in the inner stages, tA in the final
// one) are loaded with it, so the boundary path pays one memory round trip
// per plane, hidden behind the stencil.  Otherwise (16-bit storage, three
// CTAs per SM at 168 registers) the update reads FA and tA of one direction
// right before writing A (FA in the final stage) and tA, so only one
// direction's values are live; loading them early there doubled the spills.
// o0/o1: the cells' indices, m: the cells' mask.
template <int KIND, int N, bool EARLY>
struct Aux2 {
  static constexpr int NU = (KIND == 0 || !EARLY) ? 1 : N, NV = (KIND == 1 && EARLY) ? N : 1;
  f2 ai[N];
  f2 u[NU];  // EARLY: FA (inner stages) or tA (final stage)
  f2 v[NV];  // EARLY: tA (inner stages)
  __device__ __forceinline__ void load(const StageArgs &a, int d, size_t o0, size_t o1, int m,
                                       int c0) {
    const size_t as = a.g.astride[d];
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const float *b = a.ain[d] + (c0 + q) * as;
      ai[q] = ld2(b + o0, b + o1, m);
      if constexpr (EARLY && KIND == 1) {
        const float *f = a.afw[d] + (c0 + q) * as, *t = a.ta[d] + (c0 + q) * as;
        u[q] = ld2(f + o0, f + o1, m);
        v[q] = ld2(t + o0, t + o1, m);
      } else if constexpr (EARLY && KIND == 2) {
        const float *t = a.ta[d] + (c0 + q) * as;
        u[q] = ld2(t + o0, t + o1, m);
      }
    }
  }
  __device__ __forceinline__ void update(const StageArgs &a, int d, size_t o0, size_t o1, int m,
                                         int c0, const f2 *hh) const {
    const size_t as = a.g.astride[d];
    if constexpr (KIND == 0) {
#pragma unroll
      for (int q = 0; q < N; ++q) {
        float *po = a.aout[d] + (c0 + q) * as, *pt = a.ta[d] + (c0 + q) * as;
        st2(po + o0, po + o1, m, fma2(S2(a.adt), hh[q], ai[q]));
        st2(pt + o0, pt + o1, m, fma2(S2(a.bdt), hh[q], ai[q]));
      }
    } else if constexpr (EARLY) {
#pragma unroll
      for (int q = 0; q < N; ++q) {
        float *po = a.aout[d] + (c0 + q) * as, *pt = a.ta[d] + (c0 + q) * as;
        if (KIND == 1) {
          st2(po + o0, po + o1, m, fma2(S2(a.adt), hh[q], u[q]));
          st2(pt + o0, pt + o1, m, fma2(S2(a.bdt), hh[q], v[q]));
        } else {
          st2(po + o0, po + o1, m, fma2(S2(a.bdt), hh[q], u[q]));
        }
      }
    } else if constexpr (KIND == 1) {
      // FA and tA together: one memory round trip per direction
      f2 fu[N], tv[N];
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const float *b = a.afw[d] + (c0 + q) * as;
        const float *t = a.ta[d] + (c0 + q) * as;
        fu[q] = ld2(b + o0, b + o1, m);
        tv[q] = ld2(t + o0, t + o1, m);
      }
#pragma unroll
      for (int q = 0; q < N; ++q) {
        float *po = a.aout[d] + (c0 + q) * as;
        float *pt = a.ta[d] + (c0 + q) * as;
        st2(po + o0, po + o1, m, fma2(S2(a.adt), hh[q], fu[q]));
        st2(pt + o0, pt + o1, m, fma2(S2(a.bdt), hh[q], tv[q]));
      }
    } else {
      f2 tu[N];
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const float *b = a.ta[d] + (c0 + q) * as;
        tu[q] = ld2(b + o0, b + o1, m);
      }
#pragma unroll
      for (int q = 0; q < N; ++q) {
        float *po = a.aout[d] + (c0 + q) * as;
        st2(po + o0, po + o1, m, fma2(S2(a.bdt), hh[q], tu[q]));
      }
    }
  }
};

// Per-pair context of one item (tile column pair), shared by the two parts.
struct Pair {
  int i, j, ix, iy;   // first cell (valid and internal indices)
  int m;              // cells inside the grid (bit mask)
  int mx;             // cells inside an x layer (bit mask)
  bool ypml;          // the row is inside a y layer
  int xa0, xa1, ya;   // auxiliary x indices of the two cells, y index of the row
  f2 iBx, apdx, dbx, bbx;  // x profiles of the two cells (1/B, APD, DB, B)
  float iBy, apdy, dby, bby;
};

// Per-plane quantities of the general (boundary) path.
struct Plane {
  int iz, k;
  size_t c;           // linear index of the first cell
  bool zpml, top, near_top, curved, lean;
  bool met;           // the plane's metric tile was loaded
  float zz;           // zeta_z of the plane when no tile was loaded
  // zeta_z of this thread's pair
  template <typename P> __device__ __forceinline__ f2 zeta_z(const P &pw) const {
    return met ? pw.M(2) : S2(zz);
  }
};

// Pointwise operands of this thread's pair in the current slot.
template <typename T>
struct Pw2 {
  const T *u0, *u1;
  const float *coef, *met;
  __device__ f2 U0(int q) const { return ldp(u0 + q * PWT); }
  __device__ f2 U1(int q) const { return ldp(u1 + q * PWT); }
  __device__ f2 C(int q) const { return lds2(coef + q * PWT); }
  __device__ f2 M(int q) const { return lds2(met + q * PWT); }
};

// auxiliary indices of the pair on a plane (X: per cell; Y, Z: the pair is
// contiguous)
struct AuxIdx {
  size_t x0, x1, y, z;
  float iBz, apdz, dbz;
  __device__ AuxIdx() : x0(0), x1(0), y(0), z(0), iBz(1.f), apdz(0.f), dbz(0.f) {}
  __device__ AuxIdx(const StageArgs &a, const Pair &e, const Plane &pl) {
    const Geom &g = a.g;
    iBz = 1.f / a.b[2][pl.iz];
    apdz = a.apd[2][pl.iz];
    dbz = a.db[2][pl.iz];
    const size_t rx = ((size_t)pl.iz * g.nyi + e.iy) * g.nxa;
    x0 = rx + e.xa0;
    x1 = rx + e.xa1;
    y = ((size_t)pl.iz * g.nya + e.ya) * g.px + e.ix;
    const int za = (pl.k < g.nabs[4]) ? pl.k : pl.k - (g.nk - g.nabs[5]) + g.nabs[4];
    z = ((size_t)za * g.nyi + e.iy) * g.px + e.ix;
  }
};

// -------------------------- velocity part ---------------------------------
// dV/dt = (1/rho) (d_xi sigma_x + d_eta sigma_y + zeta . d_zeta sigma), each
// directional part divided by its CFS beta; ADE auxiliaries for V.  The top 3
// layers' velocities come from the traction-image kernel (timg.cu); only
// their z auxiliaries are updated here.
// w[s][q]: staged component s on plane iz + (3 - q) * Z (q = 3: this plane).
template <typename T, int X, int Y, int Z, int KIND>
__device__ __forceinline__ void vel_pair(const StageArgs &a, const Pair &e, const Plane &pl,
                                         const T *H, int ry, int cb, const Pw2<T> &pw,
                                         const typename Win<T>::type (&w)[6][5], float rx,
                                         float rys, float rz) {
  constexpr int HX = Halo<T>::HX, HPL = Halo<T>::HPL;
  const size_t fs = a.g.fstride;
  auto W = [&](int s, int q) { return Win<T>::get(w[s][q]); };
  // 1/h factors carry the staged component's scale (stored units -> values)
  auto sr = [&](float r, int s) { return scaled<T>(r, a.sc[TXX + s]); };
  auto dx = [&](int s) { return dx_pair<X>(H + s * HPL + ry * HX, cb, W(s, 3), sr(rx, s)); };
  auto dy = [&](int s) { return dy_pair<Y>(H + s * HPL, ry, cb, W(s, 3), sr(rys, s)); };
  auto dz = [&](int s) {
    return drp2(W(s, 4), W(s, 3), W(s, 2), W(s, 1), W(s, 0), sr(rz, s));
  };
  T *out = static_cast<T *>(a.out), *tw = static_cast<T *>(a.tw);
  auto adt = [&](int c) { return scaled<T>(a.adt, a.isc[c]); };
  auto bdt = [&](int c) { return scaled<T>(a.bdt, a.isc[c]); };

  if (pl.lean) {
    const f2 irho = pw.C(0);
    const f2 ztz = pl.zeta_z(pw);
    f2 hw[3];
    if (pl.curved) {
      const f2 ztx = pw.M(0), zty = pw.M(1);
      const f2 DzTxx = dz(0), DzTyy = dz(1), DzTzz = dz(2);
      const f2 DzTxy = dz(3), DzTxz = dz(4), DzTyz = dz(5);
      const f2 z0 = mul2(fma2(ztz, DzTxz, fma2(zty, DzTxy, mul2(ztx, DzTxx))), irho);
      const f2 z1 = mul2(fma2(ztz, DzTyz, fma2(zty, DzTyy, mul2(ztx, DzTxy))), irho);
      const f2 z2 = mul2(fma2(ztz, DzTzz, fma2(zty, DzTyz, mul2(ztx, DzTxz))), irho);
      hw[0] = add2(add2(mul2(dx(0), irho), mul2(dy(3), irho)), z0);
      hw[1] = add2(add2(mul2(dx(3), irho), mul2(dy(1), irho)), z1);
      hw[2] = add2(add2(mul2(dx(4), irho), mul2(dy(5), irho)), z2);
    } else {
      hw[0] = add2(add2(mul2(dx(0), irho), mul2(dy(3), irho)), mul2(mul2(ztz, dz(4)), irho));
      hw[1] = add2(add2(mul2(dx(3), irho), mul2(dy(1), irho)), mul2(mul2(ztz, dz(5)), irho));
      hw[2] = add2(add2(mul2(dx(4), irho), mul2(dy(5), irho)), mul2(mul2(ztz, dz(2)), irho));
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
      rk_store2<KIND>(a, out + (VX + q) * fs + pl.c, tw + (VX + q) * fs + pl.c, 3, pw.U0(q),
                      TwoRegs<KIND, T>::value ? pw.U1(q) : S2(0.f), hw[q], adt(VX + q), bdt(VX + q));
    return;
  }

  // general path: issue every auxiliary load before the stencil arithmetic
  const AuxIdx ix(a, e, pl);
  const int mx = e.mx, my = e.ypml ? e.m : 0, mz = pl.zpml ? e.m : 0;
  Aux2<KIND, 3, sizeof(T) == 4> ax, ay, az;
  if (mx) ax.load(a, 0, ix.x0, ix.x1, mx, 0);
  if (my) ay.load(a, 1, ix.y, ix.y + 1, my, 0);
  if (mz) az.load(a, 2, ix.z, ix.z + 1, mz, 0);
  const f2 irho = pw.C(0);
  f2 ztx = S2(0.f), zty = S2(0.f);
  const f2 ztz = pl.zeta_z(pw);
  if (pl.curved) { ztx = pw.M(0); zty = pw.M(1); }
  f2 dxi[3], det[3], dzt[3];
  dxi[0] = mul2(dx(0), irho);  // DxTxx
  dxi[1] = mul2(dx(3), irho);  // DxTxy
  dxi[2] = mul2(dx(4), irho);  // DxTxz
  det[0] = mul2(dy(3), irho);  // DyTxy
  det[1] = mul2(dy(1), irho);  // DyTyy
  det[2] = mul2(dy(5), irho);  // DyTyz
  const f2 DzTzz = dz(2), DzTxz = dz(4), DzTyz = dz(5);
  if (pl.curved) {
    const f2 DzTxx = dz(0), DzTyy = dz(1), DzTxy = dz(3);
    dzt[0] = mul2(fma2(ztz, DzTxz, fma2(zty, DzTxy, mul2(ztx, DzTxx))), irho);
    dzt[1] = mul2(fma2(ztz, DzTyz, fma2(zty, DzTyy, mul2(ztx, DzTxy))), irho);
    dzt[2] = mul2(fma2(ztz, DzTzz, fma2(zty, DzTyz, mul2(ztx, DzTxz))), irho);
  } else {
    dzt[0] = mul2(mul2(ztz, DzTxz), irho);
    dzt[1] = mul2(mul2(ztz, DzTyz), irho);
    dzt[2] = mul2(mul2(ztz, DzTzz), irho);
  }
  const f2 iBy = S2(e.iBy), iBz = S2(ix.iBz);
  f2 hw[3], hax[3], hay[3], haz[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) hw[q] = fma2(dzt[q], iBz, fma2(det[q], iBy, mul2(dxi[q], e.iBx)));
  if (mx) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      hw[q] = fma2(neg2(ax.ai[q]), e.iBx, hw[q]);
      hax[q] = fma2(neg2(e.apdx), ax.ai[q], mul2(dxi[q], e.dbx));
    }
  }
  if (my) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      hw[q] = fma2(neg2(ay.ai[q]), iBy, hw[q]);
      hay[q] = fma2(neg2(S2(e.apdy)), ay.ai[q], mul2(det[q], S2(e.dby)));
    }
  }
  if (mz) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      hw[q] = fma2(neg2(az.ai[q]), iBz, hw[q]);
      haz[q] = fma2(neg2(S2(ix.apdz)), az.ai[q], mul2(dzt[q], S2(ix.dbz)));
    }
  }
  // the top 3 layers' velocities (and their x/y auxiliaries) come from the
  // traction-image kernel; only the z auxiliaries are kept here
  const bool xy = !pl.near_top;
  const int mxs = xy ? mx : 0, mys = xy ? my : 0;
  if (mxs) ax.update(a, 0, ix.x0, ix.x1, mxs, 0, hax);
  if (mys) ay.update(a, 1, ix.y, ix.y + 1, mys, 0, hay);
  if (mz) az.update(a, 2, ix.z, ix.z + 1, mz, 0, haz);
  if (!xy) return;
#pragma unroll
  for (int q = 0; q < 3; ++q)
    rk_store2<KIND>(a, out + (VX + q) * fs + pl.c, tw + (VX + q) * fs + pl.c, e.m, pw.U0(q),
                    TwoRegs<KIND, T>::value ? pw.U1(q) : S2(0.f), hw[q], adt(VX + q), bdt(VX + q));
}

// --------------------------- stress part ----------------------------------
// dsigma/dt from Hooke's law with the velocity gradient in curvilinear form;
// the surface-layer d/dzeta of V comes from the traction-free matrices, the
// next two layers use the 2-point and Gottlieb 2-4 operators (VLOW).
// w[s][q]: velocity component s on plane iz + (3 - q) * Z.

// row r (0, 3, 6) of a surface matrix (9 planes from mv) times (u, v, t)
__device__ __forceinline__ f2 mat_row(const float *mv, size_t plane, int r, f2 u, f2 v, f2 t) {
  return fma2(lds2(mv + (r + 2) * plane), t,
              fma2(lds2(mv + (r + 1) * plane), v, mul2(lds2(mv + r * plane), u)));
}

template <typename T, int X, int Y, int Z, int KIND>
__device__ __forceinline__ void str_pair(const StageArgs &a, const Pair &e, const Plane &pl,
                                         const T *H, int ry, int cb, const Pw2<T> &pw,
                                         const typename Win<T>::type (&w)[3][5], float rx,
                                         float rys, float rz) {
  constexpr int HX = Halo<T>::HX, HPL = Halo<T>::HPL;
  const Geom &g = a.g;
  auto W = [&](int s, int q) { return Win<T>::get(w[s][q]); };
  const size_t fs = g.fstride;
  // 1/h factors carry the staged component's scale (stored units -> values)
  auto sr = [&](float r, int s) { return scaled<T>(r, a.sc[VX + s]); };
  auto dx = [&](int s) { return dx_pair<X>(H + s * HPL + ry * HX, cb, W(s, 3), sr(rx, s)); };
  auto dy = [&](int s) { return dy_pair<Y>(H + s * HPL, ry, cb, W(s, 3), sr(rys, s)); };
  auto dz = [&](int s) {
    return drp2(W(s, 4), W(s, 3), W(s, 2), W(s, 1), W(s, 0), sr(rz, s));
  };
  T *out = static_cast<T *>(a.out), *tw = static_cast<T *>(a.tw);

  // general path: issue every stage-input auxiliary load before the stencil.
  // The stress auxiliaries are kept as one per velocity derivative of the
  // direction (x: d/dx of Vx, Vy, Vz; y: d/dy; z: d/dzeta): each stress's
  // ADE auxiliary is the same linear combination of them, with cell-constant
  // coefficients, as its RHS term is of the derivatives (the ADE is linear),
  // so three values per direction stand for six.
  const bool gen = !pl.lean;
  int mx = 0, my = 0, mz = 0;
  AuxIdx ix;
  Aux2<KIND, 3, sizeof(T) == 4> ax, ay, az;
  if (gen) {
    ix = AuxIdx(a, e, pl);
    mx = e.mx;
    my = e.ypml ? e.m : 0;
    mz = pl.zpml ? e.m : 0;
    if (mx) ax.load(a, 0, ix.x0, ix.x1, mx, 3);
    if (my) ay.load(a, 1, ix.y, ix.y + 1, my, 3);
    if (mz) az.load(a, 2, ix.z, ix.z + 1, mz, 3);
  }
  const f2 DxVx = dx(0), DxVy = dx(1), DxVz = dx(2);
  const f2 DyVx = dy(0), DyVy = dy(1), DyVz = dy(2);
  f2 DzVx, DzVy, DzVz;
  // surface matrices of this pair (matVx2Vz: planes 0..8, matVy2Vz: 9..17)
  const float *mv = a.matv + (size_t)e.iy * g.px + e.ix;
  if (pl.top) {
    DzVx = add2(mat_row(mv + 9 * g.plane, g.plane, 0, DyVx, DyVy, DyVz),
                mat_row(mv, g.plane, 0, DxVx, DxVy, DxVz));
    DzVy = add2(mat_row(mv + 9 * g.plane, g.plane, 3, DyVx, DyVy, DyVz),
                mat_row(mv, g.plane, 3, DxVx, DxVy, DxVz));
    DzVz = add2(mat_row(mv + 9 * g.plane, g.plane, 6, DyVx, DyVy, DyVz),
                mat_row(mv, g.plane, 6, DxVx, DxVy, DxVz));
  } else if (pl.iz == g.top - 1) {  // 2-point (M22)
    DzVx = mul2(add2(W(0, 2), neg2(W(0, 3))), S2(sr(rz, 0)));
    DzVy = mul2(add2(W(1, 2), neg2(W(1, 3))), S2(sr(rz, 1)));
    DzVz = mul2(add2(W(2, 2), neg2(W(2, 3))), S2(sr(rz, 2)));
  } else if (pl.iz == g.top - 2) {  // Gottlieb 2-4 (M24)
    auto m24 = [&](int s) {
      return mul2(fma2(S2(CGFD_MA2), W(s, 1), fma2(S2(CGFD_MA1), W(s, 2),
                                                  mul2(S2(CGFD_MA0), W(s, 3)))), S2(sr(rz, s)));
    };
    DzVx = m24(0);
    DzVy = m24(1);
    DzVz = m24(2);
  } else {
    DzVx = dz(0);
    DzVy = dz(1);
    DzVz = dz(2);
  }

  const f2 lam2mu = pw.C(0), miu = pw.C(1);
  const f2 lambda = fma2(S2(-2.f), miu, lam2mu);
  f2 ztx = S2(0.f), zty = S2(0.f);
  const f2 ztz = pl.zeta_z(pw);
  if (pl.curved) { ztx = pw.M(0); zty = pw.M(1); }
  // components in the set order Txx Tyy Tzz Txy Txz Tyz (index q = comp - 3)
  f2 dxi[6], det[6], dzt[6];
  {
    const f2 tx2 = mul2(ztx, DzVx), ty2 = mul2(zty, DzVy), tz2 = mul2(ztz, DzVz);
    dxi[0] = mul2(lam2mu, DxVx); det[0] = mul2(lambda, DyVy);
    dzt[0] = fma2(lambda, tz2, fma2(lambda, ty2, mul2(lam2mu, tx2)));
    dxi[1] = mul2(lambda, DxVx); det[1] = mul2(lam2mu, DyVy);
    dzt[1] = fma2(lambda, tz2, fma2(lam2mu, ty2, mul2(lambda, tx2)));
    dxi[2] = mul2(lambda, DxVx); det[2] = mul2(lambda, DyVy);
    dzt[2] = fma2(lam2mu, tz2, fma2(lambda, ty2, mul2(lambda, tx2)));
    dxi[3] = mul2(DxVy, miu); det[3] = mul2(DyVx, miu);
    dzt[3] = mul2(fma2(ztx, DzVy, mul2(zty, DzVx)), miu);
    dxi[4] = mul2(DxVz, miu); det[4] = S2(0.f);
    dzt[4] = mul2(fma2(ztx, DzVz, mul2(ztz, DzVx)), miu);
    dxi[5] = S2(0.f); det[5] = mul2(DyVz, miu);
    dzt[5] = mul2(fma2(zty, DzVz, mul2(ztz, DzVy)), miu);
  }

  f2 hw[6];
  if (!gen) {
#pragma unroll
    for (int q = 0; q < 6; ++q) hw[q] = add2(add2(dxi[q], det[q]), dzt[q]);
  } else {
    const f2 iBy = S2(e.iBy), iBz = S2(ix.iBz);
#pragma unroll
    for (int q = 0; q < 6; ++q)
      hw[q] = fma2(dzt[q], iBz, fma2(det[q], iBy, mul2(dxi[q], e.iBx)));
    // surface layer: the ADE auxiliaries also take the xi (eta) part of the
    // surface-matrix d/dzeta of V (src/calculate.cu:4479-4491, 4527-4538)
    auto surf = [&](f2 z1v, f2 z2v, f2 z3v, f2 f, f2 *out) {
      const f2 a1 = mul2(ztx, z1v), a2 = mul2(zty, z2v), a3 = mul2(ztz, z3v);
      out[0] = fma2(f, fma2(lambda, a3, fma2(lambda, a2, mul2(lam2mu, a1))), out[0]);
      out[1] = fma2(f, fma2(lambda, a3, fma2(lam2mu, a2, mul2(lambda, a1))), out[1]);
      out[2] = fma2(f, fma2(lam2mu, a3, fma2(lambda, a2, mul2(lambda, a1))), out[2]);
      out[3] = fma2(f, mul2(fma2(ztx, z2v, mul2(zty, z1v)), miu), out[3]);
      out[4] = fma2(f, mul2(fma2(ztx, z3v, mul2(ztz, z1v)), miu), out[4]);
      out[5] = fma2(f, mul2(fma2(zty, z3v, mul2(ztz, z2v)), miu), out[5]);
    };
    // the six stresses' terms of a vector v of x / y / zeta derivatives of
    // (Vx, Vy, Vz), as dxi / det / dzt are of the derivatives themselves
    // (on the surface layer with the surface-matrix part, scaled by B, which
    // the auxiliary RHS of the reference carries there)
    const float *my2 = mv + 9 * g.plane;
    auto terms_x = [&](const f2 *v, f2 *o) {
      o[0] = mul2(lam2mu, v[0]); o[1] = mul2(lambda, v[0]); o[2] = mul2(lambda, v[0]);
      o[3] = mul2(v[1], miu); o[4] = mul2(v[2], miu); o[5] = S2(0.f);
      if (pl.top)
        surf(mat_row(mv, g.plane, 0, v[0], v[1], v[2]), mat_row(mv, g.plane, 3, v[0], v[1], v[2]),
             mat_row(mv, g.plane, 6, v[0], v[1], v[2]), e.bbx, o);
    };
    auto terms_y = [&](const f2 *v, f2 *o) {
      o[0] = mul2(lambda, v[1]); o[1] = mul2(lam2mu, v[1]); o[2] = mul2(lambda, v[1]);
      o[3] = mul2(v[0], miu); o[4] = S2(0.f); o[5] = mul2(v[2], miu);
      if (pl.top)
        surf(mat_row(my2, g.plane, 0, v[0], v[1], v[2]), mat_row(my2, g.plane, 3, v[0], v[1], v[2]),
             mat_row(my2, g.plane, 6, v[0], v[1], v[2]), S2(e.bby), o);
    };
    auto terms_z = [&](const f2 *v, f2 *o) {
      const f2 tx2 = mul2(ztx, v[0]), ty2 = mul2(zty, v[1]), tz2 = mul2(ztz, v[2]);
      o[0] = fma2(lambda, tz2, fma2(lambda, ty2, mul2(lam2mu, tx2)));
      o[1] = fma2(lambda, tz2, fma2(lam2mu, ty2, mul2(lambda, tx2)));
      o[2] = fma2(lam2mu, tz2, fma2(lambda, ty2, mul2(lambda, tx2)));
      o[3] = mul2(fma2(ztx, v[1], mul2(zty, v[0])), miu);
      o[4] = mul2(fma2(ztx, v[2], mul2(ztz, v[0])), miu);
      o[5] = mul2(fma2(zty, v[2], mul2(ztz, v[1])), miu);
    };
    f2 t[6];
    if (mx) {
      terms_x(ax.ai, t);
#pragma unroll
      for (int q = 0; q < 6; ++q) hw[q] = fma2(neg2(t[q]), e.iBx, hw[q]);
    }
    if (my) {
      terms_y(ay.ai, t);
#pragma unroll
      for (int q = 0; q < 6; ++q) hw[q] = fma2(neg2(t[q]), iBy, hw[q]);
    }
    if (mz) {
      terms_z(az.ai, t);
#pragma unroll
      for (int q = 0; q < 6; ++q) hw[q] = fma2(neg2(t[q]), iBz, hw[q]);
    }
    // one direction at a time: the derivative auxiliaries' RHS
    // (-APD a + DB dV), then their RK update
    f2 ha[3];
    if (mx) {
      ha[0] = fma2(neg2(e.apdx), ax.ai[0], mul2(DxVx, e.dbx));
      ha[1] = fma2(neg2(e.apdx), ax.ai[1], mul2(DxVy, e.dbx));
      ha[2] = fma2(neg2(e.apdx), ax.ai[2], mul2(DxVz, e.dbx));
      ax.update(a, 0, ix.x0, ix.x1, mx, 3, ha);
    }
    if (my) {
      ha[0] = fma2(neg2(S2(e.apdy)), ay.ai[0], mul2(DyVx, S2(e.dby)));
      ha[1] = fma2(neg2(S2(e.apdy)), ay.ai[1], mul2(DyVy, S2(e.dby)));
      ha[2] = fma2(neg2(S2(e.apdy)), ay.ai[2], mul2(DyVz, S2(e.dby)));
      ay.update(a, 1, ix.y, ix.y + 1, my, 3, ha);
    }
    if (mz) {
      ha[0] = fma2(neg2(S2(ix.apdz)), az.ai[0], mul2(DzVx, S2(ix.dbz)));
      ha[1] = fma2(neg2(S2(ix.apdz)), az.ai[1], mul2(DzVy, S2(ix.dbz)));
      ha[2] = fma2(neg2(S2(ix.apdz)), az.ai[2], mul2(DzVz, S2(ix.dbz)));
      az.update(a, 2, ix.z, ix.z + 1, mz, 3, ha);
    }
  }
  const int m = gen ? e.m : 3;
#pragma unroll
  for (int q = 0; q < 6; ++q)
    rk_store2<KIND>(a, out + (TXX + q) * fs + pl.c, tw + (TXX + q) * fs + pl.c, m, pw.U0(q),
                    TwoRegs<KIND, T>::value ? pw.U1(q) : S2(0.f), hw[q], scaled<T>(a.adt, a.isc[TXX + q]),
                    scaled<T>(a.bdt, a.isc[TXX + q]));
}

// ------------------------------ the march ---------------------------------
// items: tile index fastest, so the CTAs resident at one time work on
// neighbouring tiles of the same z-chunk and share halo rows in L2
template <typename T, int PART, int X, int Y, int Z, int KIND, bool B>
__global__ void __launch_bounds__(TT, MinCtas<T>::value)
    pair_kernel(const __grid_constant__ Maps maps, const StageArgs a, const Work wk, int *err) {
  using S = Slot<T, PART>;
  constexpr int HOFF = Halo<T>::HOFF, HX = Halo<T>::HX, HPL = Halo<T>::HPL;
  constexpr int NC = PartInfo<PART>::NC, C0 = PartInfo<PART>::C0;
  constexpr int S0 = PartInfo<PART>::S0;
  constexpr int NCOEF = PartInfo<PART>::NCOEF, COEF0 = PartInfo<PART>::COEF0;
  constexpr int DIR = (Z > 0) ? -1 : 1;  // march direction in z
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // align the ring on the shared-window address itself
  unsigned char *sbase = smem_raw + ((128u - (su32(smem_raw) & 127u)) & 127u);
  unsigned char *ring = sbase;  // NSLOT slots of S::BYTES
  uint64_t *bars = reinterpret_cast<uint64_t *>(sbase + (size_t)NSLOT * S::BYTES);
  __shared__ int abort_flag;

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;

  if (tid == 0) {
    abort_flag = 0;
    bool aligned = ((su32(bars) & 7u) == 0);
    for (int s = 0; s < NSLOT; ++s)
      aligned = aligned && ((su32(ring + (size_t)s * S::BYTES) & 127u) == 0);
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
  const int ry = ty + 3, cb = HOFF + 2 * tx;
  const int sc = ry * HX + cb;       // this pair inside a halo plane
  const int tc = ty * CX + 2 * tx;   // this pair inside a pointwise tile
  const int kinda = (KIND == 1) ? 3 : (KIND == 2 ? 2 : 1);        // aux sets read

  __shared__ int s_next;
  int base = 0;  // stream position of the current item's entry 0
  for (;;) {
    // the next item, taken only when this CTA is free (a CTA never holds a
    // claim on work while it is still busy)
    if (tid == 0) s_next = atomicAdd(wk.counter + PART, 1);
    __syncthreads();
    const int cur = s_next;
    if (cur >= wk.nitems || abort_flag) break;  // CTA-uniform
    const int4 it4 = wk.items[cur];
    const int model = B ? it4.w : 0;
    // a batched launch reads the item's model's stage arguments in place
    // (global memory, read-only during the launch).  Copied per item into a
    // __shared__ StageArgs and read from there, the 16-bit batched stages
    // behaved as if every component scale were zero (FP32, whose kernels
    // never read the scales, was unaffected); read through a pointer to the
    // copy hidden from the compiler they were correct but 15% slower than
    // in place.
    const StageArgs &A = B ? wk.bargs[model] : a;
    const Maps &M = B ? wk.bmaps[model] : maps;
    const Geom &g = A.g;
    const size_t fs = g.fstride;
    const bool flat = A.flat;
    // bytes one plane delivers: halo always, pointwise only for computed
    // planes, the metric tile only where the plane's metric is not uniform
    const uint32_t pw_bytes =
        S::U_B * (TwoRegs<KIND, T>::value ? 2u : 1u) + (uint32_t)(PWT * 4) * NCOEF;
    auto met_tile = [&](int p) { return !flat && p >= A.zu_end; };
    // zeta_z of a plane without a metric tile (loaded one plane ahead)
    auto zz_of = [&](int p) { return flat ? 1.f : (p < A.zu_end ? A.zzp[p] : 0.f); };
    const float rx = (float)X / A.h, rys = (float)Y / A.h, rz = (float)Z / A.h;
    const int zlo = LFD + g.nabs[4], zhi = g.nk + LFD - g.nabs[5];  // z interior [zlo, zhi)
    const bool aux_on[3] = {B ? A.ain[0] != nullptr : wk.has_aux[0] != 0,
                         B ? A.ain[1] != nullptr : wk.has_aux[1] != 0,
                         B ? A.ain[2] != nullptr : wk.has_aux[2] != 0};
    const int4 it = make_int4(it4.x, it4.y, it4.z & 0xffff, it4.z >> 16);
    const int i0 = it.x, j0 = it.y, z0 = it.z, z1 = it.w;
    const int n = z1 - z0;                  // planes computed (>= 4)
    const int zf = (DIR > 0) ? z0 : z1 - 1;  // first plane in march order
    // Item entries q = 0..n (plane zf + DIR*q; entry n is read for the window
    // only) go to ring slot (base + q) & 3, base counting the entries of the
    // CTA's earlier items; thread 0 issues, every thread waits, in order.
    auto issue = [&](const int4 it, int q, int s) {  // thread 0 only
      unsigned char *slot = ring + (size_t)s * S::BYTES;
      const int i0 = it.x, j0 = it.y, n = it.w - it.z;
      const int p = ((DIR > 0) ? it.z : it.w - 1) + DIR * q;
      const bool compute = q < n;
      fence_proxy_async();
      const bool met = compute && met_tile(p);
      mbar_expect_tx(&bars[s], S::HALO_B + (compute ? pw_bytes : 0u) +
                                   (met ? (uint32_t)(PWT * 4) * 3u : 0u));
      const bool withheld = PART == PART_VEL && wk.withhold == q && base == 0 &&
                            blockIdx.x == 0;
      if (!withheld) tma_load(slot, &M.halo, XO + i0 - HOFF, j0, p, C0, &bars[s]);
      if (compute) {
        const int cx = XO + i0, cy = LFD + j0;
        tma_load(slot + S::U0, &M.u0, cx, cy, p, S0, &bars[s]);
        if (TwoRegs<KIND, T>::value) tma_load(slot + S::U1, &M.u1, cx, cy, p, S0, &bars[s]);
        tma_load(slot + S::COEF, &M.coef, cx, cy, p, COEF0, &bars[s]);
        if (met) tma_load(slot + S::MET, &M.met, cx, cy, p, 0, &bars[s]);
        // the plane's PML auxiliaries into L2 (tile- and plane-uniform presence)
        const bool xp = aux_on[0] && (i0 < g.nabs[0] || i0 + CX > g.ni - g.nabs[1]);
        const bool yp = aux_on[1] && (j0 < g.nabs[2] || j0 + TY > g.nj - g.nabs[3]);
        const bool zp = aux_on[2] && (p < zlo || p >= zhi);
        if (xp || yp || zp) {
          const int xa_t = (i0 < g.nabs[0]) ? max(i0, 0) : i0 - (g.ni - g.nabs[1]) + g.xaoff;
          const int ya_t = (j0 < g.nabs[2]) ? j0 : j0 - (g.nj - g.nabs[3]) + g.nabs[2];
          const int za = (p - LFD < g.nabs[4]) ? p - LFD : p - LFD - (g.nk - g.nabs[5]) + g.nabs[4];
          const int c0 = (PART == PART_VEL) ? 0 : 3;
          const int cxp = max(cx, 0);  // prefetch boxes start inside the arrays
          for (int t = 0; t < kinda; ++t) {
            const int set = (KIND == 2 && t == 1) ? 2 : t;  // final stage: ain, ta
            if (xp) tma_prefetch(&M.aux[0][set], xa_t, cy, p, c0);
            if (yp) tma_prefetch(&M.aux[1][set], cxp, ya_t, p, c0);
            if (zp) tma_prefetch(&M.aux[2][set], cxp, cy, za, c0);
          }
        }
      }
      pend |= 1u << s;
    };

    if (tid == 0)
      for (int q = 0; q < NSLOT; ++q) issue(it, q, (base + q) & (NSLOT - 1));
    auto wait = [&](int q) -> bool {  // every thread, in march order
      const int s = (base + q) & (NSLOT - 1);
      const bool ok = mbar_wait(&bars[s], (ph >> s) & 1u, wk.wait_us);
      if (ok) {  // an expired wait leaves the copy pending for the drain
        ph ^= 1u << s;
        if (tid == 0) pend &= ~(1u << s);
      }
      return ok;
    };

    Pair e;
    e.i = i0 + 2 * tx;
    e.j = j0 + ty;
    e.ix = e.i + XO;
    e.iy = e.j + LFD;
    const bool rowok = e.j < g.nj;  // (tile origins may lie left of the grid)
    e.m = (rowok && e.i >= 0 && e.i < g.ni ? 1 : 0) | (rowok && e.i + 1 >= 0 && e.i + 1 < g.ni ? 2 : 0);
    auto inx = [&](int i) { return i < g.nabs[0] || i >= g.ni - g.nabs[1]; };
    e.mx = ((e.m & 1) && inx(e.i) ? 1 : 0) | ((e.m & 2) && inx(e.i + 1) ? 2 : 0);
    e.ypml = e.m && (e.j < g.nabs[2] || e.j >= g.nj - g.nabs[3]);
    // xa1 = xa0 + 1 whenever both cells are in a layer (xaoff), and xa0 is
    // even then, so the pair is one aligned 64-bit access
    auto xa = [&](int i) { return (i < g.nabs[0]) ? i : i - (g.ni - g.nabs[1]) + g.xaoff; };
    e.xa0 = xa(e.i);
    e.xa1 = xa(e.i + 1);
    e.ya = (e.j < g.nabs[2]) ? e.j : e.j - (g.nj - g.nabs[3]) + g.nabs[2];
    e.iBx = S2(1.f); e.apdx = S2(0.f); e.dbx = S2(0.f); e.bbx = S2(1.f);
    e.iBy = 1.f; e.apdy = 0.f; e.dby = 0.f; e.bby = 1.f;
    if (e.m & 1) {
      e.bbx.x = A.b[0][e.ix]; e.iBx.x = 1.f / e.bbx.x;
      e.apdx.x = A.apd[0][e.ix]; e.dbx.x = A.db[0][e.ix];
    }
    if (e.m & 2) {
      e.bbx.y = A.b[0][e.ix + 1]; e.iBx.y = 1.f / e.bbx.y;
      e.apdx.y = A.apd[0][e.ix + 1]; e.dbx.y = A.db[0][e.ix + 1];
    }
    if (e.m) {
      e.bby = A.b[1][e.iy]; e.iBy = 1.f / e.bby;
      e.apdy = A.apd[1][e.iy]; e.dby = A.db[1][e.iy];
    }
    // tile-uniform: no x/y PML anywhere in this tile (and B = 1, DB = APD = 0
    // outside the layers, which the solver checks at upload)
    const bool tile_int = A.plain_interior && (i0 >= g.nabs[0]) &&
                          (i0 + CX <= g.ni - g.nabs[1]) && (j0 >= g.nabs[2]) &&
                          (j0 + TY <= g.nj - g.nabs[3]);

    // register window: w[c][q] = plane (current) + DIR * (q - 3)
    typename Win<T>::type w[NC][5];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int q = 0; q < 5; ++q) w[c][q] = Win<T>::zero();
    auto push_smem = [&](const unsigned char *slot) {
      const T *plane = reinterpret_cast<const T *>(slot);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
#pragma unroll
        for (int q = 0; q < 4; ++q) w[c][q] = w[c][q + 1];
        w[c][4] = Win<T>::ld(plane + c * HPL + sc);
      }
    };
    // the three planes behind the chunk come straight from global memory
    for (int k = 3; k >= 1; --k) {
      const size_t o = gidx(g, e.ix, e.iy, zf - DIR * k);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
#pragma unroll
        for (int q = 0; q < 4; ++q) w[c][q] = w[c][q + 1];
        const T *src = static_cast<const T *>(A.in) + (size_t)(C0 + c) * fs + o;
        w[c][4] = e.m ? Win<T>::ldm(src, e.m) : Win<T>::zero();
      }
    }
    // A wait that expires sets the CTA-wide abort flag; the flag is read only
    // after a __syncthreads, so every thread leaves the march together.
    if (wait(0)) push_smem(ring + (size_t)(base & (NSLOT - 1)) * S::BYTES);
    else abort_flag = 1;
    __syncthreads();

    size_t c = gidx(g, e.ix, e.iy, zf);
    float zzn = zz_of(zf);
#pragma unroll MARCH_UNROLL
    for (int q = 0; q < n; ++q) {
      const float zzc = zzn;
      if (q + 1 < n) zzn = zz_of(zf + DIR * (q + 1));
      const bool got = wait(q + 1);
      if (got) push_smem(ring + (size_t)((base + q + 1) & (NSLOT - 1)) * S::BYTES);
      else abort_flag = 1;
      if (e.m && got) {
        const unsigned char *slot = ring + (size_t)((base + q) & (NSLOT - 1)) * S::BYTES;
        Plane pl;
        pl.iz = zf + DIR * q;
        pl.k = pl.iz - LFD;
        pl.c = c;
        pl.top = (pl.iz == g.top);
        pl.near_top = pl.iz >= g.top - 2;
        pl.zpml = (pl.iz < zlo) || (pl.iz >= zhi);
        pl.curved = pl.iz >= g.con && !flat;
        pl.lean = tile_int && !pl.zpml && !pl.near_top;
        pl.met = met_tile(pl.iz);
        pl.zz = zzc;
        const Pw2<T> pw{reinterpret_cast<const T *>(slot + S::U0) + tc,
                        reinterpret_cast<const T *>(slot + S::U1) + tc,
                        reinterpret_cast<const float *>(slot + S::COEF) + tc,
                        reinterpret_cast<const float *>(slot + S::MET) + tc};
        const T *H = reinterpret_cast<const T *>(slot);
        if constexpr (PART == PART_VEL)
          vel_pair<T, X, Y, Z, KIND>(A, e, pl, H, ry, cb, pw, w, rx, rys, rz);
        else
          str_pair<T, X, Y, Z, KIND>(A, e, pl, H, ry, cb, pw, w, rx, rys, rz);
      }
      // the slot of entry q is free: refill it with stream position
      // base + q + NSLOT (this item's entry q + 4, or the next item's)
      __syncthreads();
      if (abort_flag) break;
      if (tid == 0 && q + NSLOT <= n) issue(it, q + NSLOT, (base + q) & (NSLOT - 1));
      c += (DIR > 0) ? g.plane : (size_t)0 - g.plane;
    }
    __syncthreads();  // all reads of the ring done before the next item reuses it
    base += n + 1;
  }
  if (abort_flag && tid == 0) {
    if (err) atomicExch(err, 1);
    // drain: wait (bounded) for copies still in flight before the CTA's
    // shared memory goes away
    for (int s = 0; s < NSLOT; ++s)
      if (pend & (1u << s)) mbar_wait(&bars[s], (ph >> s) & 1u, wk.wait_us);
  }
}

// Tensor maps of one model's buffers (host side, stage_pair.cu): per field
// set (FW, Wa, Wb, tW) the halo boxes of the two parts and the pointwise
// boxes of V (3) and T (6) components; media, metric; auxiliaries per
// direction and set (FA, A, tA) for V and T components.
struct ModelMaps {
  CUtensorMap haloV[4], haloS[4], ctrV[4], ctrT[4];
  CUtensorMap coefV, coefS, met;
  CUtensorMap auxV[3][3], auxT[3][3];
};

// Launch plan of one solver or of a batch of models.
struct Plan {
  std::vector<ModelMaps> mm;   // one per model
  std::vector<Geom> geoms;
  Work wk;
  int elem;                    // storage element type of the field sets
  int zchunk;                  // planes of the (first model's) interior z-chunks
  int grid[2];
  WorkParams params;
  int nmodels = 0;             // 0: single-model plan; else a batch of nmodels
  StageArgs *d_bargs = nullptr;  // batch: [pattern * 4 + stage][model]
  Maps *d_bmaps = nullptr;       // batch: [stage][part][model]
};

// a: the single model's stage arguments (X, Y, Z and the stage kind come
// from it in every case); a batched launch (B) takes each model's arguments
// and maps from pl.wk instead
template <typename T, int PART, int X, int Y, int Z, int KIND, bool B>
void launch_t(const Plan &pl, const Maps &m, const StageArgs &a, const Work &wk, int *err,
              cudaStream_t s) {
  pair_kernel<T, PART, X, Y, Z, KIND, B>
      <<<pl.grid[PART], dim3(TX, TY, 1), Slot<T, PART>::SMEM, s>>>(m, a, wk, err);
}

template <typename T, int PART, int KIND, bool B = false>
void launch_dirs(const Plan &pl, const Maps &m, const StageArgs &a, const Work &wk, int *err,
                 cudaStream_t s) {
  const int code = (a.X > 0 ? 4 : 0) + (a.Y > 0 ? 2 : 0) + (a.Z > 0 ? 1 : 0);
  switch (code) {
    case 0: launch_t<T, PART, -1, -1, -1, KIND, B>(pl, m, a, wk, err, s); break;
    case 1: launch_t<T, PART, -1, -1, 1, KIND, B>(pl, m, a, wk, err, s); break;
    case 2: launch_t<T, PART, -1, 1, -1, KIND, B>(pl, m, a, wk, err, s); break;
    case 3: launch_t<T, PART, -1, 1, 1, KIND, B>(pl, m, a, wk, err, s); break;
    case 4: launch_t<T, PART, 1, -1, -1, KIND, B>(pl, m, a, wk, err, s); break;
    case 5: launch_t<T, PART, 1, -1, 1, KIND, B>(pl, m, a, wk, err, s); break;
    case 6: launch_t<T, PART, 1, 1, -1, KIND, B>(pl, m, a, wk, err, s); break;
    default: launch_t<T, PART, 1, 1, 1, KIND, B>(pl, m, a, wk, err, s); break;
  }
}

template <typename T, int PART, int KIND, bool B = false>
void set_attrs() {
  auto set = [](const void *f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Slot<T, PART>::SMEM);
  };
  set((const void *)pair_kernel<T, PART, -1, -1, -1, KIND, B>);
  set((const void *)pair_kernel<T, PART, -1, -1, 1, KIND, B>);
  set((const void *)pair_kernel<T, PART, -1, 1, -1, KIND, B>);
  set((const void *)pair_kernel<T, PART, -1, 1, 1, KIND, B>);
  set((const void *)pair_kernel<T, PART, 1, -1, -1, KIND, B>);
  set((const void *)pair_kernel<T, PART, 1, -1, 1, KIND, B>);
  set((const void *)pair_kernel<T, PART, 1, 1, -1, KIND, B>);
  set((const void *)pair_kernel<T, PART, 1, 1, 1, KIND, B>);
}

template <typename T, int PART, bool B = false>
int resident_ctas() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pair_kernel<T, PART, 1, 1, 1, 1, B>, TT,
                                                Slot<T, PART>::SMEM);
  if (per < 1) per = 1;
  if (sms < 1) sms = 1;
  return per * sms;
}

// per-(storage, part, kind) entry points, one translation unit each
// (pair_{f,h,b}{v,s}{0,1,2}.cu; f: FP32, h: FP16, b: BF16 storage), each
// with its batched kernels (suffix _b)
#define CGFD_PAIR_DECL(E, P, K)                                                          \
  void launch_##E##P##K(const Plan &pl, const Maps &m, const StageArgs &a, int *err,   \
                        cudaStream_t s);                                                \
  void attrs_##E##P##K();
#define CGFD_PAIR_DECL_B(E, P, K)                                                        \
  void launch_##E##P##K##_b(const Plan &pl, const StageArgs &a, const Work &wk, int *err, \
                            cudaStream_t s);                                            \
  void attrs_##E##P##K##_b();
#define CGFD_PAIR_DECL_E(E)                                                   \
  CGFD_PAIR_DECL(E, v, 0) CGFD_PAIR_DECL(E, v, 1) CGFD_PAIR_DECL(E, v, 2)     \
  CGFD_PAIR_DECL(E, s, 0) CGFD_PAIR_DECL(E, s, 1) CGFD_PAIR_DECL(E, s, 2)     \
  int resident_##E##v();                                                      \
  int resident_##E##s();
CGFD_PAIR_DECL_E(f)
CGFD_PAIR_DECL_E(h)
CGFD_PAIR_DECL_E(b)
#define CGFD_PAIR_DECL_BE(E)                                                         \
  CGFD_PAIR_DECL_B(E, v, 0) CGFD_PAIR_DECL_B(E, v, 1) CGFD_PAIR_DECL_B(E, v, 2)          \
  CGFD_PAIR_DECL_B(E, s, 0) CGFD_PAIR_DECL_B(E, s, 1) CGFD_PAIR_DECL_B(E, s, 2)          \
  int resident_##E##v_b();                                                            \
  int resident_##E##s_b();
CGFD_PAIR_DECL_BE(f)
CGFD_PAIR_DECL_BE(h)
CGFD_PAIR_DECL_BE(b)
#undef CGFD_PAIR_DECL_BE
#undef CGFD_PAIR_DECL_B
#undef CGFD_PAIR_DECL_E
#undef CGFD_PAIR_DECL

}  // namespace pair
}  // namespace cgfd
