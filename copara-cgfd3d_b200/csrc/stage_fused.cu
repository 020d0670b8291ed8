// stage_fused.cu -- z-marching tiled RK stage kernels for sm_100a.
//
// One RK stage is two kernels, split along the velocity-stress structure of
// the equations: the velocity part needs only stress derivatives and the
// stress part only velocity derivatives, so each kernel stages only the
// components it differentiates and carries half the register state.
//
// Each CTA owns a 32 x 4 tile of (x, y) columns and marches upwards through a
// chunk of z-planes.  Per plane, the differentiated components of the stage
// input arrive with an x/y halo by TMA (cp.async.bulk.tensor, one 4-D box
// {40 x, 10 y, 1 z, NC components} per plane, no multicast) into a ring of 5
// shared-memory slots, one mbarrier per slot, so the loads of the next planes
// overlap the arithmetic on the current one.  The one-sided DRP stencils reach
// -1..+3 or -3..+1 cells; the box covers -4..+4 in x (x origin 16-byte
// aligned) and -3..+3 in y.  z stencils run from per-thread register windows
// of 5 planes per component.  The RK update (Iteration*), the CFS-PML
// auxiliaries and the free-surface work (VLOW operators, surface matrices,
// traction image) are fused into the same pass: a stage reads W_in once from
// HBM for its stencils plus FW / tW / aux and the coefficients, and writes
// W_out / tW / aux.  There are no derivative or hW arrays.
//
// Per cell the arithmetic is that of the reference's CalDiffmix + CalWavemix
// + CalTIMGmix + Iteration* (src/calculate.cu:4121-4621, 5668-5897,
// 6330-6734); point sources are added by a separate tiny kernel (solver.cu).
//
// Every wait on an mbarrier is bounded (about 2 s of %globaltimer).  On
// expiry the CTA leaves the march together (the flag is read after a
// barrier), records an error code in *err, waits (bounded) for its own copies
// still in flight and returns; the host then reports CGFD_ERR_TIMEOUT.
#include "cgfd_internal.cuh"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

namespace cgfd {
namespace {

constexpr int TX = 32, TY = 4;                 // threads per CTA tile
constexpr int BOXX = TX + 8, BOXY = TY + 6;    // TMA box (x starts 4 left, y 3 below)
constexpr int NSLOT = 5;
constexpr int PLANE = BOXX * BOXY;             // floats per component per plane
constexpr unsigned long long WAIT_NS = 2000000000ull;
enum { PART_VEL = 0, PART_STR = 1 };

template <int PART> struct PartInfo;
template <> struct PartInfo<PART_VEL> {  // stresses are staged
  static constexpr int NC = 6, C0 = TXX;
};
template <> struct PartInfo<PART_STR> {  // velocities are staged
  static constexpr int NC = 3, C0 = VX;
};
// bytes one TMA box delivers, and the slot stride: a tensor copy needs a
// 128-byte aligned shared-memory destination, so slots are padded to 128 B
template <int PART>
__host__ __device__ constexpr uint32_t box_bytes() { return (uint32_t)(PLANE * PartInfo<PART>::NC * 4); }
template <int PART>
__host__ __device__ constexpr uint32_t slot_bytes() { return (box_bytes<PART>() + 127u) / 128u * 128u; }
// ring + barriers, plus 128 B of slack to align the ring base
template <int PART>
__host__ __device__ constexpr size_t smem_bytes() { return (size_t)NSLOT * slot_bytes<PART>() + 128 + 128; }
static_assert(slot_bytes<0>() % 128 == 0 && slot_bytes<1>() % 128 == 0, "slot alignment");

__device__ __forceinline__ uint32_t su32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// bounded wait; false on expiry
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity) {
  if (mbar_try_wait(b, parity)) return true;
  const unsigned long long t0 = gtime();
  while (!mbar_try_wait(b, parity))
    if (gtime() - t0 > WAIT_NS) return false;
  return true;
}
__device__ __forceinline__ void tma_load(float *dst, const CUtensorMap *map, int x, int y, int z,
                                         int c, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(su32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(su32(bar))
      : "memory");
}

__device__ __forceinline__ float drp5(float m1, float c0, float p1, float p2, float p3, float r) {
  return (CGFD_DA_1 * m1 + CGFD_DA0 * c0 + CGFD_DA1 * p1 + CGFD_DA2 * p2 + CGFD_DA3 * p3) * r;
}

// RK update of one value (Iteration*): KIND 0 first stage, 1 inner, 2 final
template <int KIND>
__device__ __forceinline__ void rk_put(float *out, float *tw, const float *fw, size_t o, float fwv,
                                       float hh, float adt, float bdt) {
  if (KIND == 0) {
    out[o] = fwv + adt * hh;
    tw[o] = fwv + bdt * hh;
  } else if (KIND == 1) {
    out[o] = fw[o] + adt * hh;
    tw[o] = tw[o] + bdt * hh;
  } else {
    out[o] = tw[o] + bdt * hh;
  }
}

// Per-cell context shared by the two parts.
struct Cell {
  int i, j, k, ix, iy, iz;
  size_t c;          // linear index
  bool top, near_top, zpml, xpml, ypml, interior;
  float iBx, iBy, iBz;
  size_t px, py, pz;  // aux indices
};

// -------------------------- velocity part ---------------------------------
// dV/dt = (1/rho) (d_xi sigma_x + d_eta sigma_y + zeta . d_zeta sigma), each
// directional part divided by its CFS beta; ADE auxiliaries for V; traction
// image for the top 3 layers.
template <int X, int Y, int Z, int KIND, int LAG>
__device__ __forceinline__ void vel_cell(const StageArgs &a, const Cell &e, const float *P,
                                         int sc, const float (&w)[6][5], float rx, float ry,
                                         float rz) {
  const Geom &g = a.g;
  const size_t fs = g.fstride;
  // staged components: 0 Txx 1 Tyy 2 Tzz 3 Txy 4 Txz 5 Tyz
  auto xs = [&](int s, int d) { return P[s * PLANE + sc + X * d]; };
  auto ys = [&](int s, int d) { return P[s * PLANE + sc + Y * d * BOXX]; };
  auto zs = [&](int s, int d) { return w[s][LAG + Z * d]; };
  auto dx = [&](int s) { return drp5(xs(s, -1), xs(s, 0), xs(s, 1), xs(s, 2), xs(s, 3), rx); };
  auto dy = [&](int s) { return drp5(ys(s, -1), ys(s, 0), ys(s, 1), ys(s, 2), ys(s, 3), ry); };
  auto dz = [&](int s) { return drp5(zs(s, -1), zs(s, 0), zs(s, 1), zs(s, 2), zs(s, 3), rz); };

  const float irho = a.irho[e.c];
  float ztx = 0.f, zty = 0.f, ztz = 1.f;
  const bool curved = e.iz >= g.con && !a.flat;
  if (!a.flat) {
    ztz = a.zz[e.c];
    if (curved) { ztx = a.zx[e.c]; zty = a.zy[e.c]; }
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
    for (int q = 0; q < 3; ++q) hw[q] = dxi[q] * e.iBx + det[q] * e.iBy + dzt[q] * e.iBz;
    float hax[3], hay[3], haz[3];
    if (e.xpml) {
      const float APD = a.apd[0][e.ix], DB = a.db[0][e.ix];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const float av = a.ain[0][q * g.astride[0] + e.px];
        hw[q] -= av * e.iBx;
        hax[q] = dxi[q] * DB - APD * av;
      }
    }
    if (e.ypml) {
      const float APD = a.apd[1][e.iy], DB = a.db[1][e.iy];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const float av = a.ain[1][q * g.astride[1] + e.py];
        hw[q] -= av * e.iBy;
        hay[q] = det[q] * DB - APD * av;
      }
    }
    if (e.zpml) {
      const float APD = a.apd[2][e.iz], DB = a.db[2][e.iz];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const float av = a.ain[2][q * g.astride[2] + e.pz];
        hw[q] -= av * e.iBz;
        haz[q] = dzt[q] * DB - APD * av;
      }
    }
    if (e.near_top) {
      // traction image (CalTIMGmix): conservative momentum equation with the
      // normal traction J zeta.sigma odd about the surface; the z vector is
      // read from global memory since it reaches 3 planes to either side
      const int s = g.top - e.iz;
      const float rhojac = a.flat ? irho : irho / a.jac[e.c];
      const long sy = g.px, sz = (long)g.plane;
      constexpr int TS[3][2] = {{0, 3}, {3, 1}, {4, 5}};  // staged (x, y) stress per V
      constexpr int TC[3][3] = {{TXX, TXY, TXZ}, {TXY, TYY, TYZ}, {TXZ, TYZ, TZZ}};
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        float vx[5], vy[5], vz[7];
#pragma unroll
        for (int d = -1; d <= 3; ++d) {
          float jx = 1.f, jy = 1.f;
          if (!a.flat) {
            jx = a.jac[(long)e.c + X * d];
            jy = a.jac[(long)e.c + Y * d * sy];
          }
          vx[d + 1] = jx * xs(TS[q][0], d);
          vy[d + 1] = jy * ys(TS[q][1], d);
        }
#pragma unroll
        for (int n = 0; n < 7; ++n) {
          const long gz = (long)e.c + (n - 3) * sz;
          const float t1 = a.in[TC[q][0] * fs + gz], t2 = a.in[TC[q][1] * fs + gz],
                      t3 = a.in[TC[q][2] * fs + gz];
          vz[n] = a.flat ? t3 : a.jac[gz] * (a.zx[gz] * t1 + a.zy[gz] * t2 + a.zz[gz] * t3);
        }
        // the surface is s layers up (vector index 3+s): zero there, odd above
        if (s == 0) {
          vz[3] = 0.f; vz[4] = -vz[2]; vz[5] = -vz[1]; vz[6] = -vz[0];
        } else if (s == 1) {
          vz[4] = 0.f; vz[5] = -vz[3]; vz[6] = -vz[2];
        } else {
          vz[5] = 0.f; vz[6] = -vz[4];
        }
        const float DxT = rhojac * drp5(vx[0], vx[1], vx[2], vx[3], vx[4], rx);
        const float DyT = rhojac * drp5(vy[0], vy[1], vy[2], vy[3], vy[4], ry);
        const float DzT = rhojac * drp5(vz[3 - Z], vz[3], vz[3 + Z], vz[3 + 2 * Z], vz[3 + 3 * Z], rz);
        float hv = DxT * e.iBx + DyT * e.iBy + DzT;
        if (e.xpml) {
          const float av = a.ain[0][q * g.astride[0] + e.px];
          hv -= av * e.iBx;
          hax[q] = a.db[0][e.ix] * DxT - a.apd[0][e.ix] * av;
        }
        if (e.ypml) {
          const float av = a.ain[1][q * g.astride[1] + e.py];
          hv -= av * e.iBy;
          hay[q] = a.db[1][e.iy] * DyT - a.apd[1][e.iy] * av;
        }
        hw[q] = hv;
      }
    }
    auto aux = [&](int d, size_t p, const float *hh) {
      const size_t as = g.astride[d];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const size_t o = q * as + p;
        rk_put<KIND>(a.aout[d], a.ta[d], a.afw[d], o, KIND == 0 ? a.ain[d][o] : 0.f, hh[q],
                     a.adt, a.bdt);
      }
    };
    if (e.xpml) aux(0, e.px, hax);
    if (e.ypml) aux(1, e.py, hay);
    if (e.zpml) aux(2, e.pz, haz);
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const size_t o = (size_t)(VX + q) * fs + e.c;
    rk_put<KIND>(a.out, a.tw, a.fw, o, KIND == 0 ? a.in[o] : 0.f, hw[q], a.adt, a.bdt);
  }
}

// --------------------------- stress part ----------------------------------
// dsigma/dt from Hooke's law with the velocity gradient in curvilinear form;
// the surface-layer d/dzeta of V comes from the traction-free matrices, the
// next two layers use the 2-point and Gottlieb 2-4 operators (VLOW).
template <int X, int Y, int Z, int KIND, int LAG>
__device__ __forceinline__ void str_cell(const StageArgs &a, const Cell &e, const float *P,
                                         int sc, const float (&w)[3][5], float rx, float ry,
                                         float rz) {
  const Geom &g = a.g;
  const size_t fs = g.fstride;
  auto xs = [&](int s, int d) { return P[s * PLANE + sc + X * d]; };
  auto ys = [&](int s, int d) { return P[s * PLANE + sc + Y * d * BOXX]; };
  auto zs = [&](int s, int d) { return w[s][LAG + Z * d]; };
  auto dx = [&](int s) { return drp5(xs(s, -1), xs(s, 0), xs(s, 1), xs(s, 2), xs(s, 3), rx); };
  auto dy = [&](int s) { return drp5(ys(s, -1), ys(s, 0), ys(s, 1), ys(s, 2), ys(s, 3), ry); };
  auto dz = [&](int s) { return drp5(zs(s, -1), zs(s, 0), zs(s, 1), zs(s, 2), zs(s, 3), rz); };

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

  const float lam2mu = a.lam2mu[e.c], miu = a.mu[e.c];
  const float lambda = lam2mu - 2.f * miu;
  float ztx = 0.f, zty = 0.f, ztz = 1.f;
  if (!a.flat) {
    ztz = a.zz[e.c];
    if (e.iz >= g.con) { ztx = a.zx[e.c]; zty = a.zy[e.c]; }
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
    for (int q = 0; q < 6; ++q) hw[q] = dxi[q] * e.iBx + det[q] * e.iBy + dzt[q] * e.iBz;
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
        const float av = a.ain[0][(3 + q) * g.astride[0] + e.px];
        hw[q] -= av * e.iBx;
        hax[q] = dxi[q] * DB - APD * av;
      }
      if (e.top)
        surf(cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz, cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz,
             cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz, DB * a.b[0][e.ix], hax);
    }
    if (e.ypml) {
      const float APD = a.apd[1][e.iy], DB = a.db[1][e.iy];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const float av = a.ain[1][(3 + q) * g.astride[1] + e.py];
        hw[q] -= av * e.iBy;
        hay[q] = det[q] * DB - APD * av;
      }
      if (e.top)
        surf(cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz, cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz,
             cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz, DB * a.b[1][e.iy], hay);
    }
    if (e.zpml) {
      const float APD = a.apd[2][e.iz], DB = a.db[2][e.iz];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const float av = a.ain[2][(3 + q) * g.astride[2] + e.pz];
        hw[q] -= av * e.iBz;
        haz[q] = dzt[q] * DB - APD * av;
      }
    }
    auto aux = [&](int d, size_t p, const float *hh) {
      const size_t as = g.astride[d];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const size_t o = (3 + q) * as + p;
        rk_put<KIND>(a.aout[d], a.ta[d], a.afw[d], o, KIND == 0 ? a.ain[d][o] : 0.f, hh[q],
                     a.adt, a.bdt);
      }
    };
    if (e.xpml) aux(0, e.px, hax);
    if (e.ypml) aux(1, e.py, hay);
    if (e.zpml) aux(2, e.pz, haz);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const size_t o = (size_t)(TXX + q) * fs + e.c;
    rk_put<KIND>(a.out, a.tw, a.fw, o, KIND == 0 ? a.in[o] : 0.f, hw[q], a.adt, a.bdt);
  }
}

// ------------------------------ the march ---------------------------------
template <int PART, int X, int Y, int Z, int KIND>
__global__ void __launch_bounds__(TX *TY, 4)
    stage_part_kernel(const __grid_constant__ CUtensorMap tmap, const StageArgs a, int zchunk,
                      int *err) {
  constexpr int NC = PartInfo<PART>::NC, C0 = PartInfo<PART>::C0;
  constexpr uint32_t SB = slot_bytes<PART>(), BB = box_bytes<PART>();
  constexpr int SLOTF = SB / 4;  // float stride between slots
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // align the ring on the shared-window address itself
  unsigned char *base = smem_raw + ((128u - (su32(smem_raw) & 127u)) & 127u);
  float *ring = reinterpret_cast<float *>(base);
  uint64_t *bars = reinterpret_cast<uint64_t *>(base + (size_t)NSLOT * SB);
  __shared__ int abort_flag;

  const Geom &g = a.g;
  constexpr int LEAD = (Z > 0) ? 3 : 1, LAG = (Z > 0) ? 1 : 3;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int bx0 = blockIdx.x * TX, by0 = blockIdx.y * TY;
  Cell e;
  e.i = bx0 + tx;
  e.j = by0 + ty;
  const bool active = (e.i < g.ni) && (e.j < g.nj);
  e.ix = e.i + XO;
  e.iy = e.j + LFD;
  const int z0 = LFD + blockIdx.z * zchunk;
  const int z1 = min(z0 + zchunk, g.nk + LFD);
  const int pmax = z1 - 1 + LEAD;  // last plane the chunk reads
  const size_t fs = g.fstride;

  int issued = z0 - 1;  // last plane whose load thread 0 has issued
  if (tid == 0) {
    abort_flag = 0;
    // self-check before any copy is issued: 128-byte aligned slot
    // destinations, 8-byte aligned barriers, 16-byte aligned box origin
    bool aligned = ((su32(bars) & 7u) == 0) && ((bx0 * 4) % 16 == 0);
    for (int s = 0; s < NSLOT; ++s) aligned = aligned && ((su32(ring + (size_t)s * SLOTF) & 127u) == 0);
    if (!aligned) {
      abort_flag = 1;
      if (err) atomicExch(err, 2);
    } else {
      for (int s = 0; s < NSLOT; ++s) mbar_init(&bars[s], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      for (int p = z0; p < z0 + NSLOT && p <= pmax; ++p) {
        const int s = p % NSLOT;
        mbar_expect_tx(&bars[s], BB);
        tma_load(ring + (size_t)s * SLOTF, &tmap, bx0, by0, p, C0, &bars[s]);
        issued = p;
      }
    }
  }
  __syncthreads();
  if (abort_flag) return;  // nothing was issued

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
  const int sc = (ty + 3) * BOXX + (tx + 4);  // this column inside a slot plane
  // planes below the chunk come straight from global memory (centre only)
  for (int p = z0 - LAG; p < z0; ++p) {
    if (active) push(a.in + (size_t)C0 * fs, fs, gidx(g, e.ix, e.iy, p));
    else push(ring, 0, 0);  // keeps the window shape; values unused
  }
  // A wait that expires sets the CTA-wide abort flag; the flag is read only
  // after a __syncthreads, so every thread leaves the march together.
  for (int p = z0; p < z0 + LEAD; ++p) {
    const int s = p % NSLOT;
    if (mbar_wait(&bars[s], ((p - z0) / NSLOT) & 1)) push(ring + (size_t)s * SLOTF, PLANE, sc);
    else abort_flag = 1;
  }
  __syncthreads();

  const float rx = (float)X / a.h, ry = (float)Y / a.h, rz = (float)Z / a.h;
  e.xpml = active && (e.i < g.nabs[0] || e.i >= g.ni - g.nabs[1]);
  e.ypml = active && (e.j < g.nabs[2] || e.j >= g.nj - g.nabs[3]);
  const int xa = (e.i < g.nabs[0]) ? e.i : e.i - (g.ni - g.nabs[1]) + g.nabs[0];
  const int ya = (e.j < g.nabs[2]) ? e.j : e.j - (g.nj - g.nabs[3]) + g.nabs[2];
  e.iBx = 1.f / a.b[0][e.ix];
  e.iBy = 1.f / a.b[1][e.iy];
  // tile-uniform: no x/y PML anywhere in this tile (and B = 1, DB = APD = 0
  // outside the layers, which the solver checks at upload)
  const bool tile_xy_interior =
      a.plain_interior && (bx0 >= g.nabs[0]) && (bx0 + TX <= g.ni - g.nabs[1]) &&
      (by0 >= g.nabs[2]) && (by0 + TY <= g.nj - g.nabs[3]);

  for (int iz = z0; iz < z1 && !abort_flag; ++iz) {
    bool got;
    {  // bring plane iz+LEAD into the windows
      const int p = iz + LEAD, s = p % NSLOT;
      got = mbar_wait(&bars[s], ((p - z0) / NSLOT) & 1);
      if (got) push(ring + (size_t)s * SLOTF, PLANE, sc);
      else abort_flag = 1;
    }
    if (active && got) {
      const float *P = ring + (size_t)(iz % NSLOT) * SLOTF;  // plane iz with halo
      e.iz = iz;
      e.k = iz - LFD;
      e.c = gidx(g, e.ix, e.iy, iz);
      e.top = (iz == g.top);
      e.near_top = iz >= g.top - 2;
      e.zpml = (e.k < g.nabs[4]) || (e.k >= g.nk - g.nabs[5]);
      e.interior = tile_xy_interior && !e.zpml && !e.near_top;
      e.iBz = 1.f / a.b[2][iz];
      e.px = ((size_t)iz * g.nyi + e.iy) * g.nxa + xa;
      e.py = ((size_t)iz * g.nya + ya) * g.px + e.ix;
      const int za = (e.k < g.nabs[4]) ? e.k : e.k - (g.nk - g.nabs[5]) + g.nabs[4];
      e.pz = ((size_t)za * g.nyi + e.iy) * g.px + e.ix;
      if constexpr (PART == PART_VEL)
        vel_cell<X, Y, Z, KIND, LAG>(a, e, P, sc, w, rx, ry, rz);
      else
        str_cell<X, Y, Z, KIND, LAG>(a, e, P, sc, w, rx, ry, rz);
    }
    // the slot of plane iz is free: refill it with plane iz+NSLOT
    __syncthreads();
    if (abort_flag) break;
    if (tid == 0 && iz + NSLOT <= pmax) {
      const int p = iz + NSLOT, s = p % NSLOT;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&bars[s], BB);
      tma_load(ring + (size_t)s * SLOTF, &tmap, bx0, by0, p, C0, &bars[s]);
      issued = p;
    }
  }
  __syncthreads();
  if (abort_flag && tid == 0) {
    if (err) atomicExch(err, 1);
    // drain: wait (bounded) for the copies still possibly in flight (at most
    // one per slot) before the CTA's shared memory goes away
    for (int p = max(z0, issued - NSLOT + 1); p <= issued; ++p)
      mbar_wait(&bars[p % NSLOT], ((p - z0) / NSLOT) & 1);
  }
}

// ------------------------------ host side ---------------------------------

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

// 4-D map over one field set: {x: px, y: nyi, z: nzi, component: 9}, box of
// nc components
bool make_map(CUtensorMap *m, const Geom &g, const float *base, int nc) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)g.px, (cuuint64_t)g.nyi, (cuuint64_t)g.nzi, 9};
  cuuint64_t strides[3] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.plane * 4,
                           (cuuint64_t)g.fstride * 4};
  cuuint32_t box[4] = {BOXX, BOXY, 1, (cuuint32_t)nc};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int PART, int X, int Y, int Z, int KIND>
void launch_t(const CUtensorMap &m, const StageArgs &a, int zchunk, int *err, cudaStream_t s) {
  const int nzc = (a.g.nk + zchunk - 1) / zchunk;
  dim3 grid((a.g.ni + TX - 1) / TX, (a.g.nj + TY - 1) / TY, nzc);
  stage_part_kernel<PART, X, Y, Z, KIND>
      <<<grid, dim3(TX, TY, 1), smem_bytes<PART>(), s>>>(m, a, zchunk, err);
}

template <int PART, int KIND>
void launch_dirs(const CUtensorMap &m, const StageArgs &a, int zc, int *err, cudaStream_t s) {
  const int code = (a.X > 0 ? 4 : 0) + (a.Y > 0 ? 2 : 0) + (a.Z > 0 ? 1 : 0);
  switch (code) {
    case 0: launch_t<PART, -1, -1, -1, KIND>(m, a, zc, err, s); break;
    case 1: launch_t<PART, -1, -1, 1, KIND>(m, a, zc, err, s); break;
    case 2: launch_t<PART, -1, 1, -1, KIND>(m, a, zc, err, s); break;
    case 3: launch_t<PART, -1, 1, 1, KIND>(m, a, zc, err, s); break;
    case 4: launch_t<PART, 1, -1, -1, KIND>(m, a, zc, err, s); break;
    case 5: launch_t<PART, 1, -1, 1, KIND>(m, a, zc, err, s); break;
    case 6: launch_t<PART, 1, 1, -1, KIND>(m, a, zc, err, s); break;
    default: launch_t<PART, 1, 1, 1, KIND>(m, a, zc, err, s); break;
  }
}

template <int PART>
void launch_part(const CUtensorMap &m, const StageArgs &a, int zc, int *err, cudaStream_t s) {
  if (a.rk == 0) launch_dirs<PART, 0>(m, a, zc, err, s);
  else if (a.rk < 3) launch_dirs<PART, 1>(m, a, zc, err, s);
  else launch_dirs<PART, 2>(m, a, zc, err, s);
}

template <int PART, int KIND>
void set_attrs() {
  auto set = [](const void *f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem_bytes<PART>());
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

}  // namespace

bool fused_supported(const Geom &g) {
  // the tile's TMA box starts on a 16-byte boundary (XO = 4 floats, px a
  // multiple of 32) and the grid is at least one chunk deep
  return (XO % 4) == 0 && g.px % 32 == 0 && g.nk >= 4;
}

size_t fused_map_bytes() { return 2 * sizeof(CUtensorMap); }

bool fused_make_map(void *map, const Geom &g, const float *set_base) {
  CUtensorMap *m = reinterpret_cast<CUtensorMap *>(map);
  return make_map(&m[0], g, set_base, PartInfo<PART_VEL>::NC) &&
         make_map(&m[1], g, set_base, PartInfo<PART_STR>::NC);
}

int fused_zchunk(const Geom &g) {
  // enough CTAs for ~4 per SM on 148 SMs, chunks of at least 16 planes
  const long tiles = (long)((g.ni + TX - 1) / TX) * ((g.nj + TY - 1) / TY);
  int nzc = (int)((4L * 148 + tiles - 1) / tiles);
  nzc = nzc < 1 ? 1 : nzc;
  int zc = (g.nk + nzc - 1) / nzc;
  if (zc < 16) zc = 16;
  if (zc > g.nk) zc = g.nk;
  return zc;
}

void fused_init_attributes() {
  set_attrs<PART_VEL, 0>(); set_attrs<PART_VEL, 1>(); set_attrs<PART_VEL, 2>();
  set_attrs<PART_STR, 0>(); set_attrs<PART_STR, 1>(); set_attrs<PART_STR, 2>();
}

void launch_stage_fused_map(const void *map, const StageArgs &a, int zchunk, int *err,
                            void *stream) {
  const CUtensorMap *m = reinterpret_cast<const CUtensorMap *>(map);
  cudaStream_t s = (cudaStream_t)stream;
  launch_part<PART_VEL>(m[0], a, zchunk, err, s);
  launch_part<PART_STR>(m[1], a, zchunk, err, s);
}

}  // namespace cgfd
