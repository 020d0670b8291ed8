// stage_fused.cu -- z-marching tiled RK stage kernel for sm_100a.
//
// One CTA owns a 32 x 4 tile of (x, y) columns and marches upwards through a
// chunk of z-planes.  For every plane it needs the 9 wavefield components of
// the stage input with an x/y halo (the one-sided DRP stencils reach -1..+3
// or -3..+1 cells); those arrive by TMA (cp.async.bulk.tensor, one 4-D box
// {40 x, 10 y, 1 z, 9 components} per plane, no multicast) into a ring of 5
// shared-memory slots, completed on one mbarrier per slot, so the loads of
// the next planes overlap the arithmetic of the current one.  The z stencils
// run from a per-thread register window of 5 planes per component.  The RK
// update (Iteration*), the CFS-PML auxiliaries and the free-surface work (VLOW
// operators, surface matrices, traction image) are fused into the same pass,
// so a stage reads W_in (once from HBM), FW / tW / aux and the coefficients,
// and writes W_out / tW / aux: no derivative or hW arrays exist.
//
// Semantics per cell are those of the reference's CalDiffmix + CalWavemix +
// CalTIMGmix + Iteration* (src/calculate.cu:4121-4621, 5668-5897, 6330-6734);
// point sources are added by a separate tiny kernel (solver.cu).
//
// Every wait on an mbarrier is bounded (about 2 s of %globaltimer); on
// expiry the kernel records an error code in *err, waits (bounded) for its
// own copies still in flight and returns, so the host reports
// CGFD_ERR_TIMEOUT instead of the GPU hanging.
#include "cgfd_internal.cuh"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdio>

namespace cgfd {
namespace {

constexpr int TX = 32, TY = 4;                 // threads per CTA tile
constexpr int BOXX = TX + 8, BOXY = TY + 6;    // TMA box (x starts 4 left, y 3 below)
constexpr int NSLOT = 5;
constexpr int PLANE = BOXX * BOXY;             // floats per component per plane
constexpr int SLOT = PLANE * NCOMP;            // floats per slot
constexpr uint32_t SLOT_BYTES = SLOT * 4;
constexpr size_t SMEM_BYTES = (size_t)NSLOT * SLOT_BYTES + 128;  // + barriers
constexpr unsigned long long WAIT_NS = 2000000000ull;

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
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(su32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(su32(bar))
      : "memory");
}

__device__ __forceinline__ float drp5(float m1, float c0, float p1, float p2, float p3, float r) {
  return (CGFD_DA_1 * m1 + CGFD_DA0 * c0 + CGFD_DA1 * p1 + CGFD_DA2 * p2 + CGFD_DA3 * p3) * r;
}

// KIND: 0 = first stage (in = FW), 1 = inner stages, 2 = final stage
template <int X, int Y, int Z, int KIND>
__global__ void __launch_bounds__(TX *TY, 3)
    stage_fused_kernel(const __grid_constant__ CUtensorMap tmap, const StageArgs a, int zchunk,
                       int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *ring = reinterpret_cast<float *>(smem_raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)NSLOT * SLOT_BYTES);
  __shared__ int abort_flag;

  const Geom &g = a.g;
  constexpr int LEAD = (Z > 0) ? 3 : 1, LAG = (Z > 0) ? 1 : 3;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int bx0 = blockIdx.x * TX, by0 = blockIdx.y * TY;
  const int i = bx0 + tx, j = by0 + ty;  // valid-cell indices
  const bool active = (i < g.ni) && (j < g.nj);
  const int ix = i + XO, iy = j + LFD;
  const int z0 = LFD + blockIdx.z * zchunk;
  const int z1 = min(z0 + zchunk, g.nk + LFD);
  const int pmax = z1 - 1 + LEAD;  // last plane the chunk reads
  const size_t fs = g.fstride;

  int issued = z0 - 1;  // last plane whose load thread 0 has issued
  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < NSLOT; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int p = z0; p < z0 + NSLOT && p <= pmax; ++p) {
      const int s = p % NSLOT;
      mbar_expect_tx(&bars[s], SLOT_BYTES);
      tma_load(ring + (size_t)s * SLOT, &tmap, bx0, by0, p, &bars[s]);
      issued = p;
    }
  }
  __syncthreads();

  // register windows: w[c][0..4] = planes iz-LAG .. iz+LEAD at this column
  float w[NCOMP][5];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c)
#pragma unroll
    for (int q = 0; q < 5; ++q) w[c][q] = 0.f;
  auto push = [&](const float *src, size_t stride, size_t off) {
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
#pragma unroll
      for (int q = 0; q < 4; ++q) w[c][q] = w[c][q + 1];
      w[c][4] = src[c * stride + off];
    }
  };
  const int sc = (ty + 3) * BOXX + (tx + 4);  // this column inside a slot plane
  // planes below the chunk come straight from global memory (centre only)
  for (int p = z0 - LAG; p < z0; ++p) {
    if (active) push(a.in, fs, gidx(g, ix, iy, p));
    else push(ring, 0, 0);  // keeps the window shape; values unused
  }
  // A wait that expires sets the CTA-wide abort flag; the flag is read only
  // after a __syncthreads, so every thread leaves the march together.
  for (int p = z0; p < z0 + LEAD; ++p) {
    const int s = p % NSLOT;
    if (mbar_wait(&bars[s], ((p - z0) / NSLOT) & 1)) push(ring + (size_t)s * SLOT, PLANE, sc);
    else abort_flag = 1;
  }
  __syncthreads();

  // per-column constants
  const float rx = (float)X / a.h, ry = (float)Y / a.h, rz = (float)Z / a.h;
  const bool xpml = active && (i < g.nabs[0] || i >= g.ni - g.nabs[1]);
  const bool ypml = active && (j < g.nabs[2] || j >= g.nj - g.nabs[3]);
  const int xa = (i < g.nabs[0]) ? i : i - (g.ni - g.nabs[1]) + g.nabs[0];
  const int ya = (j < g.nabs[2]) ? j : j - (g.nj - g.nabs[3]) + g.nabs[2];
  const float Bx = a.b[0][ix], By = a.b[1][iy];
  const float iBx = 1.f / Bx, iBy = 1.f / By;
  const float APDx = a.apd[0][ix], DBx = a.db[0][ix], APDy = a.apd[1][iy], DBy = a.db[1][iy];
  // tile-uniform: no x/y PML anywhere in this tile (and B = 1, DB = APD = 0
  // outside the layers, which the solver checks at upload)
  const bool tile_xy_interior =
      a.plain_interior && (bx0 >= g.nabs[0]) && (bx0 + TX <= g.ni - g.nabs[1]) &&
      (by0 >= g.nabs[2]) && (by0 + TY <= g.nj - g.nabs[3]);

  for (int iz = z0; iz < z1 && !abort_flag; ++iz) {
    // bring plane iz+LEAD into the windows
    bool got;
    {
      const int p = iz + LEAD, s = p % NSLOT;
      got = mbar_wait(&bars[s], ((p - z0) / NSLOT) & 1);
      if (got) push(ring + (size_t)s * SLOT, PLANE, sc);
      else abort_flag = 1;
    }
    const float *P = ring + (size_t)(iz % NSLOT) * SLOT;  // plane iz with halo
    if (active && got) {
      const int k = iz - LFD;
      const size_t cidx = gidx(g, ix, iy, iz);
      auto xs = [&](int c, int d) { return P[c * PLANE + sc + X * d]; };
      auto ys = [&](int c, int d) { return P[c * PLANE + sc + Y * d * BOXX]; };
      auto zs = [&](int c, int d) { return w[c][LAG + Z * d]; };
      auto dx = [&](int c) { return drp5(xs(c, -1), xs(c, 0), xs(c, 1), xs(c, 2), xs(c, 3), rx); };
      auto dy = [&](int c) { return drp5(ys(c, -1), ys(c, 0), ys(c, 1), ys(c, 2), ys(c, 3), ry); };
      auto dz = [&](int c) { return drp5(zs(c, -1), zs(c, 0), zs(c, 1), zs(c, 2), zs(c, 3), rz); };

      const float DxTxx = dx(TXX), DxTxy = dx(TXY), DxTxz = dx(TXZ);
      const float DxVx = dx(VX), DxVy = dx(VY), DxVz = dx(VZ);
      const float DyTyy = dy(TYY), DyTxy = dy(TXY), DyTyz = dy(TYZ);
      const float DyVx = dy(VX), DyVy = dy(VY), DyVz = dy(VZ);
      const float DzTzz = dz(TZZ), DzTxz = dz(TXZ), DzTyz = dz(TYZ);
      const bool curved = iz >= g.con;
      float DzTxx = 0.f, DzTyy = 0.f, DzTxy = 0.f;
      if (curved && !a.flat) { DzTxx = dz(TXX); DzTyy = dz(TYY); DzTxy = dz(TXY); }
      const bool top = (iz == g.top);
      float DzVx, DzVy, DzVz;
      float cx[9], cy[9];
      if (top) {
        const size_t m2 = (size_t)iy * g.px + ix;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          cx[q] = a.matv[q * g.plane + m2];
          cy[q] = a.matv[(9 + q) * g.plane + m2];
        }
        DzVx = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz + cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz;
        DzVy = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz + cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz;
        DzVz = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz + cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz;
      } else if (iz == g.top - 1) {  // 2-point (M22)
        DzVx = (zs(VX, 1) - zs(VX, 0)) * rz;
        DzVy = (zs(VY, 1) - zs(VY, 0)) * rz;
        DzVz = (zs(VZ, 1) - zs(VZ, 0)) * rz;
      } else if (iz == g.top - 2) {  // Gottlieb 2-4 (M24)
        DzVx = (CGFD_MA0 * zs(VX, 0) + CGFD_MA1 * zs(VX, 1) + CGFD_MA2 * zs(VX, 2)) * rz;
        DzVy = (CGFD_MA0 * zs(VY, 0) + CGFD_MA1 * zs(VY, 1) + CGFD_MA2 * zs(VY, 2)) * rz;
        DzVz = (CGFD_MA0 * zs(VZ, 0) + CGFD_MA1 * zs(VZ, 1) + CGFD_MA2 * zs(VZ, 2)) * rz;
      } else {
        DzVx = dz(VX); DzVy = dz(VY); DzVz = dz(VZ);
      }

      const float lam2mu = a.lam2mu[cidx], miu = a.mu[cidx], irho = a.irho[cidx];
      const float lambda = lam2mu - 2.f * miu;
      float ztx = 0.f, zty = 0.f, ztz = 1.f;
      if (!a.flat) {
        ztz = a.zz[cidx];
        if (curved) { ztx = a.zx[cidx]; zty = a.zy[cidx]; }
      }
      float dxi[9], det[9], dzt[9];
      dxi[VX] = DxTxx * irho; det[VX] = DyTxy * irho; dzt[VX] = (ztx * DzTxx + zty * DzTxy + ztz * DzTxz) * irho;
      dxi[VY] = DxTxy * irho; det[VY] = DyTyy * irho; dzt[VY] = (ztx * DzTxy + zty * DzTyy + ztz * DzTyz) * irho;
      dxi[VZ] = DxTxz * irho; det[VZ] = DyTyz * irho; dzt[VZ] = (ztx * DzTxz + zty * DzTyz + ztz * DzTzz) * irho;
      dxi[TXX] = lam2mu * DxVx; det[TXX] = lambda * DyVy;
      dzt[TXX] = lam2mu * ztx * DzVx + lambda * zty * DzVy + lambda * ztz * DzVz;
      dxi[TYY] = lambda * DxVx; det[TYY] = lam2mu * DyVy;
      dzt[TYY] = lambda * ztx * DzVx + lam2mu * zty * DzVy + lambda * ztz * DzVz;
      dxi[TZZ] = lambda * DxVx; det[TZZ] = lambda * DyVy;
      dzt[TZZ] = lambda * ztx * DzVx + lambda * zty * DzVy + lam2mu * ztz * DzVz;
      dxi[TXY] = DxVy * miu; det[TXY] = DyVx * miu; dzt[TXY] = (zty * DzVx + ztx * DzVy) * miu;
      dxi[TXZ] = DxVz * miu; det[TXZ] = 0.f;        dzt[TXZ] = (ztz * DzVx + ztx * DzVz) * miu;
      dxi[TYZ] = 0.f;        det[TYZ] = DyVz * miu; dzt[TYZ] = (ztz * DzVy + zty * DzVz) * miu;

      const bool zpml = (k < g.nabs[4]) || (k >= g.nk - g.nabs[5]);
      const bool near_top = iz >= g.top - 2;
      float hw[9];
      if (tile_xy_interior && !zpml && !near_top) {
        // interior: B = 1, no auxiliaries
#pragma unroll
        for (int q = 0; q < 9; ++q) hw[q] = dxi[q] + det[q] + dzt[q];
      } else {
        const float Bz = a.b[2][iz], iBz = 1.f / Bz;
#pragma unroll
        for (int q = 0; q < 9; ++q) hw[q] = dxi[q] * iBx + det[q] * iBy + dzt[q] * iBz;
        float hax[9], hay[9], haz[9];
        size_t px_ = 0, py_ = 0, pz_ = 0;
        if (xpml) {
          px_ = ((size_t)iz * g.nyi + iy) * g.nxa + xa;
          const size_t as = g.astride[0];
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            const float av = a.ain[0][q * as + px_];
            hw[q] -= av * iBx;
            hax[q] = dxi[q] * DBx - APDx * av;
          }
          if (top) {
            const float z1v = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz;
            const float z2v = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz;
            const float z3v = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz;
            const float f = DBx * Bx;
            hax[TXX] += f * (lam2mu * ztx * z1v + lambda * zty * z2v + lambda * ztz * z3v);
            hax[TYY] += f * (lambda * ztx * z1v + lam2mu * zty * z2v + lambda * ztz * z3v);
            hax[TZZ] += f * (lambda * ztx * z1v + lambda * zty * z2v + lam2mu * ztz * z3v);
            hax[TXY] += f * (zty * z1v + ztx * z2v) * miu;
            hax[TXZ] += f * (ztz * z1v + ztx * z3v) * miu;
            hax[TYZ] += f * (ztz * z2v + zty * z3v) * miu;
          }
        }
        if (ypml) {
          py_ = ((size_t)iz * g.nya + ya) * g.px + ix;
          const size_t as = g.astride[1];
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            const float av = a.ain[1][q * as + py_];
            hw[q] -= av * iBy;
            hay[q] = det[q] * DBy - APDy * av;
          }
          if (top) {
            const float z1v = cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz;
            const float z2v = cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz;
            const float z3v = cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz;
            const float f = DBy * By;
            hay[TXX] += f * (lam2mu * ztx * z1v + lambda * zty * z2v + lambda * ztz * z3v);
            hay[TYY] += f * (lambda * ztx * z1v + lam2mu * zty * z2v + lambda * ztz * z3v);
            hay[TZZ] += f * (lambda * ztx * z1v + lambda * zty * z2v + lam2mu * ztz * z3v);
            hay[TXY] += f * (zty * z1v + ztx * z2v) * miu;
            hay[TXZ] += f * (ztz * z1v + ztx * z3v) * miu;
            hay[TYZ] += f * (ztz * z2v + zty * z3v) * miu;
          }
        }
        if (zpml) {
          const int za = (k < g.nabs[4]) ? k : k - (g.nk - g.nabs[5]) + g.nabs[4];
          pz_ = ((size_t)za * g.nyi + iy) * g.px + ix;
          const size_t as = g.astride[2];
          const float APDz = a.apd[2][iz], DBz = a.db[2][iz];
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            const float av = a.ain[2][q * as + pz_];
            hw[q] -= av * iBz;
            haz[q] = dzt[q] * DBz - APDz * av;
          }
        }
        if (near_top) {
          // traction image for the velocities (CalTIMGmix); the z vector is
          // read from global memory since it reaches 3 planes to either side
          const int s = g.top - iz;
          const float rhojac = a.flat ? irho : irho / a.jac[cidx];
          const long sx = 1, sy = g.px, sz = (long)g.plane;
          constexpr int TC[3][3] = {{TXX, TXY, TXZ}, {TXY, TYY, TYZ}, {TXZ, TYZ, TZZ}};
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            float vx[5], vy[5], vz[7];
#pragma unroll
            for (int d = -1; d <= 3; ++d) {
              float jx = 1.f, jy = 1.f;
              if (!a.flat) {
                jx = a.jac[(long)cidx + X * d * sx];
                jy = a.jac[(long)cidx + Y * d * sy];
              }
              vx[d + 1] = jx * xs(TC[q][0], d);
              vy[d + 1] = jy * ys(TC[q][1], d);
            }
#pragma unroll
            for (int n = 0; n < 7; ++n) {
              const long gz = (long)cidx + (n - 3) * sz;
              const float t1 = a.in[TC[q][0] * fs + gz], t2 = a.in[TC[q][1] * fs + gz],
                          t3 = a.in[TC[q][2] * fs + gz];
              vz[n] = a.flat ? t3 : a.jac[gz] * (a.zx[gz] * t1 + a.zy[gz] * t2 + a.zz[gz] * t3);
            }
#pragma unroll
            for (int p = 1; p <= LFD; ++p)
              if (p <= LFD - s) vz[3 + s + p] = -vz[3 + s - p];
            vz[3 + s] = 0.f;
            const float DxT = rhojac * drp5(vx[0], vx[1], vx[2], vx[3], vx[4], rx);
            const float DyT = rhojac * drp5(vy[0], vy[1], vy[2], vy[3], vy[4], ry);
            const float DzT = rhojac * drp5(vz[3 - Z], vz[3], vz[3 + Z], vz[3 + 2 * Z], vz[3 + 3 * Z], rz);
            float hv = DxT * iBx + DyT * iBy + DzT;
            if (xpml) {
              const float av = a.ain[0][q * g.astride[0] + px_];
              hv -= av * iBx;
              hax[q] = DBx * DxT - APDx * av;
            }
            if (ypml) {
              const float av = a.ain[1][q * g.astride[1] + py_];
              hv -= av * iBy;
              hay[q] = DBy * DyT - APDy * av;
            }
            hw[q] = hv;
          }
        }
        // auxiliary RK update (each value read and written by its own thread)
        auto aux = [&](int d, size_t p, const float *hh) {
          const size_t as = g.astride[d];
          float *ao = a.aout[d], *ta = a.ta[d];
#pragma unroll
          for (int q = 0; q < 9; ++q) {
            const size_t o = q * as + p;
            if (KIND == 0) {
              const float f = a.ain[d][o];
              ao[o] = f + a.adt * hh[q];
              ta[o] = f + a.bdt * hh[q];
            } else if (KIND == 1) {
              ao[o] = a.afw[d][o] + a.adt * hh[q];
              ta[o] = ta[o] + a.bdt * hh[q];
            } else {
              ao[o] = ta[o] + a.bdt * hh[q];
            }
          }
        };
        if (xpml) aux(0, px_, hax);
        if (ypml) aux(1, py_, hay);
        if (zpml) aux(2, pz_, haz);
      }

      // RK update of the wavefield (Iteration*)
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        const size_t o = q * fs + cidx;
        if (KIND == 0) {
          const float f = zs(q, 0);  // FW is the stage input
          a.out[o] = f + a.adt * hw[q];
          a.tw[o] = f + a.bdt * hw[q];
        } else if (KIND == 1) {
          a.out[o] = a.fw[o] + a.adt * hw[q];
          a.tw[o] = a.tw[o] + a.bdt * hw[q];
        } else {
          a.out[o] = a.tw[o] + a.bdt * hw[q];
        }
      }
    }
    // slot of plane iz is free: refill it with plane iz+NSLOT
    __syncthreads();
    if (abort_flag) break;
    if (tid == 0 && iz + NSLOT <= pmax) {
      const int p = iz + NSLOT, s = p % NSLOT;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&bars[s], SLOT_BYTES);
      tma_load(ring + (size_t)s * SLOT, &tmap, bx0, by0, p, &bars[s]);
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

// 4-D map over one field set: {x: px, y: nyi, z: nzi, component: 9}
bool make_map(CUtensorMap *m, const Geom &g, const float *base) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)g.px, (cuuint64_t)g.nyi, (cuuint64_t)g.nzi, 9};
  cuuint64_t strides[3] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.plane * 4,
                           (cuuint64_t)g.fstride * 4};
  cuuint32_t box[4] = {BOXX, BOXY, 1, NCOMP};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int X, int Y, int Z, int KIND>
void launch_t(const CUtensorMap &m, const StageArgs &a, int zchunk, int *err, cudaStream_t s) {
  auto k = stage_fused_kernel<X, Y, Z, KIND>;
  const int nzc = (a.g.nk + zchunk - 1) / zchunk;
  dim3 grid((a.g.ni + TX - 1) / TX, (a.g.nj + TY - 1) / TY, nzc);
  k<<<grid, dim3(TX, TY, 1), SMEM_BYTES, s>>>(m, a, zchunk, err);
}

template <int KIND>
void launch_dirs(const CUtensorMap &m, const StageArgs &a, int zc, int *err, cudaStream_t s) {
  const int code = (a.X > 0 ? 4 : 0) + (a.Y > 0 ? 2 : 0) + (a.Z > 0 ? 1 : 0);
  switch (code) {
    case 0: launch_t<-1, -1, -1, KIND>(m, a, zc, err, s); break;
    case 1: launch_t<-1, -1, 1, KIND>(m, a, zc, err, s); break;
    case 2: launch_t<-1, 1, -1, KIND>(m, a, zc, err, s); break;
    case 3: launch_t<-1, 1, 1, KIND>(m, a, zc, err, s); break;
    case 4: launch_t<1, -1, -1, KIND>(m, a, zc, err, s); break;
    case 5: launch_t<1, -1, 1, KIND>(m, a, zc, err, s); break;
    case 6: launch_t<1, 1, -1, KIND>(m, a, zc, err, s); break;
    default: launch_t<1, 1, 1, KIND>(m, a, zc, err, s); break;
  }
}

}  // namespace

bool fused_supported(const Geom &g) {
  // the tile's TMA box must start on a 16-byte boundary (XO = 4 floats) and
  // the grid must be at least one chunk deep
  return (XO % 4) == 0 && g.px % 4 == 0 && g.nk >= 4;
}

size_t fused_map_bytes() { return sizeof(CUtensorMap); }

bool fused_make_map(void *map, const Geom &g, const float *set_base) {
  return make_map(reinterpret_cast<CUtensorMap *>(map), g, set_base);
}

int fused_zchunk(const Geom &g) {
  // enough CTAs for ~3 per SM on 148 SMs, chunks of at least 16 planes
  const long tiles = (long)((g.ni + TX - 1) / TX) * ((g.nj + TY - 1) / TY);
  int nzc = (int)((3L * 148 * 2 + tiles - 1) / tiles);
  nzc = nzc < 1 ? 1 : nzc;
  int zc = (g.nk + nzc - 1) / nzc;
  if (zc < 16) zc = 16;
  if (zc > g.nk) zc = g.nk;
  return zc;
}

void launch_stage_fused_map(const void *map, const StageArgs &a, int zchunk, int *err,
                            void *stream) {
  const CUtensorMap &m = *reinterpret_cast<const CUtensorMap *>(map);
  cudaStream_t s = (cudaStream_t)stream;
  if (a.rk == 0) launch_dirs<0>(m, a, zchunk, err, s);
  else if (a.rk < 3) launch_dirs<1>(m, a, zchunk, err, s);
  else launch_dirs<2>(m, a, zchunk, err, s);
}

void fused_init_attributes() {
  auto set = [](const void *f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  };
#define CGFD_ATTR(K)                                                                       \
  set((const void *)stage_fused_kernel<-1, -1, -1, K>);                                   \
  set((const void *)stage_fused_kernel<-1, -1, 1, K>);                                    \
  set((const void *)stage_fused_kernel<-1, 1, -1, K>);                                    \
  set((const void *)stage_fused_kernel<-1, 1, 1, K>);                                     \
  set((const void *)stage_fused_kernel<1, -1, -1, K>);                                    \
  set((const void *)stage_fused_kernel<1, -1, 1, K>);                                     \
  set((const void *)stage_fused_kernel<1, 1, -1, K>);                                     \
  set((const void *)stage_fused_kernel<1, 1, 1, K>);
  CGFD_ATTR(0)
  CGFD_ATTR(1)
  CGFD_ATTR(2)
#undef CGFD_ATTR
}

}  // namespace cgfd
