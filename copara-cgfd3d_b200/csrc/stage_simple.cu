// stage_simple.cu -- one-thread-per-cell RK stage kernel.
//
// A direct, untiled statement of one RK stage on the internal layout: every
// thread reads its stencils straight from global memory (through L1/L2),
// computes the RHS of its cell and applies the RK update.  It is kept as the
// on-GPU cross-check of the tiled z-marching kernel (stage_fused.cu) and is
// selectable with CGFD_KERNEL_SIMPLE.
//
// Per cell it does the work of the reference's
//   CalDiffmix  src/calculate.cu:4121-4275  (DRP/M22/M24 + surface matrices)
//   CalWavemix  src/calculate.cu:4277-4621  (Hooke/momentum RHS, ADE CFS-PML)
//   CalTIMGmix  src/calculate.cu:5668-5897  (traction image, top 3 layers)
//   Iteration*  src/calculate.cu:6330-6734  (RK4 update of fields and aux)
// without the 27 derivative arrays and the hW array of the reference.
#include "cgfd_internal.cuh"

#include <cuda_runtime.h>

namespace cgfd {
namespace {

__device__ __forceinline__ float drp(const float *v, long g, long s, int d, float rh) {
  const long ds = d * s;
  return (CGFD_DA_1 * v[g - ds] + CGFD_DA0 * v[g] + CGFD_DA1 * v[g + ds] +
          CGFD_DA2 * v[g + 2 * ds] + CGFD_DA3 * v[g + 3 * ds]) * rh;
}
__device__ __forceinline__ float m22(const float *v, long g, long s, int d, float rh) {
  return (v[g + d * s] - v[g]) * rh;
}
__device__ __forceinline__ float m24(const float *v, long g, long s, int d, float rh) {
  const long ds = d * s;
  return (CGFD_MA0 * v[g] + CGFD_MA1 * v[g + ds] + CGFD_MA2 * v[g + 2 * ds]) * rh;
}
__device__ __forceinline__ float strf7(const float *v, int d, float rh) {
  return (CGFD_DA_1 * v[3 - d] + CGFD_DA0 * v[3] + CGFD_DA1 * v[3 + d] +
          CGFD_DA2 * v[3 + 2 * d] + CGFD_DA3 * v[3 + 3 * d]) * rh;
}

template <int RK>
__device__ __forceinline__ void rk_update(float hh, float fwv, float &outv, float &twv,
                                          float adt, float bdt) {
  if (RK == 0) {
    outv = fwv + adt * hh;
    twv = fwv + bdt * hh;
  } else if (RK < 3) {
    outv = fwv + adt * hh;
    twv = twv + bdt * hh;
  } else {
    outv = twv + bdt * hh;
  }
}

template <int RK>
__global__ void __launch_bounds__(128) stage_simple_kernel(StageArgs a) {
  const Geom &g = a.g;
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = blockIdx.y * 4 + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.ni || j >= g.nj) return;
  const int ix = i + XO, iy = j + LFD, iz = k + LFD;
  const long c = (long)gidx(g, ix, iy, iz);
  const long sx = 1, sy = g.px, sz = (long)g.plane;
  const size_t fs = g.fstride;
  const float *in = static_cast<const float *>(a.in);  // FP32 storage only
  const float *Vx = in + VX * fs, *Vy = in + VY * fs, *Vz = in + VZ * fs;
  const float *Txx = in + TXX * fs, *Tyy = in + TYY * fs, *Tzz = in + TZZ * fs;
  const float *Txy = in + TXY * fs, *Txz = in + TXZ * fs, *Tyz = in + TYZ * fs;
  const float rx = a.X / a.h, ry = a.Y / a.h, rz = a.Z / a.h;

  // ---- directional derivatives (CalDiffmix) ----
  const float DxTxx = drp(Txx, c, sx, a.X, rx), DxTxy = drp(Txy, c, sx, a.X, rx),
              DxTxz = drp(Txz, c, sx, a.X, rx), DxVx = drp(Vx, c, sx, a.X, rx),
              DxVy = drp(Vy, c, sx, a.X, rx), DxVz = drp(Vz, c, sx, a.X, rx);
  const float DyTyy = drp(Tyy, c, sy, a.Y, ry), DyTxy = drp(Txy, c, sy, a.Y, ry),
              DyTyz = drp(Tyz, c, sy, a.Y, ry), DyVx = drp(Vx, c, sy, a.Y, ry),
              DyVy = drp(Vy, c, sy, a.Y, ry), DyVz = drp(Vz, c, sy, a.Y, ry);
  const float DzTzz = drp(Tzz, c, sz, a.Z, rz), DzTxz = drp(Txz, c, sz, a.Z, rz),
              DzTyz = drp(Tyz, c, sz, a.Z, rz);
  const bool curved = iz >= g.con;
  float DzTxx = 0.f, DzTyy = 0.f, DzTxy = 0.f;
  if (curved) {
    DzTxx = drp(Txx, c, sz, a.Z, rz);
    DzTyy = drp(Tyy, c, sz, a.Z, rz);
    DzTxy = drp(Txy, c, sz, a.Z, rz);
  }
  const size_t m2 = (size_t)iy * g.px + ix;
  float cx[9], cy[9];
  float DzVx, DzVy, DzVz;
  if (iz == g.top) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      cx[q] = a.matv[q * g.plane + m2];
      cy[q] = a.matv[(9 + q) * g.plane + m2];
    }
    DzVx = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz + cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz;
    DzVy = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz + cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz;
    DzVz = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz + cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz;
  } else if (iz == g.top - 1) {
    DzVx = m22(Vx, c, sz, a.Z, rz); DzVy = m22(Vy, c, sz, a.Z, rz); DzVz = m22(Vz, c, sz, a.Z, rz);
  } else if (iz == g.top - 2) {
    DzVx = m24(Vx, c, sz, a.Z, rz); DzVy = m24(Vy, c, sz, a.Z, rz); DzVz = m24(Vz, c, sz, a.Z, rz);
  } else {
    DzVx = drp(Vx, c, sz, a.Z, rz); DzVy = drp(Vy, c, sz, a.Z, rz); DzVz = drp(Vz, c, sz, a.Z, rz);
  }

  // ---- RHS (CalWavemix) ----
  const float lam2mu = a.lam2mu[c], miu = a.mu[c], irho = a.irho[c];
  const float lambda = lam2mu - 2.f * miu;
  float ztx = 0.f, zty = 0.f, ztz = 1.f;
  if (!a.flat) {
    ztz = a.zz[c];
    if (curved) { ztx = a.zx[c]; zty = a.zy[c]; }
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

  const float Bx = a.b[0][ix], By = a.b[1][iy], Bz = a.b[2][iz];
  float hw[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) hw[q] = dxi[q] / Bx + det[q] / By + dzt[q] / Bz;

  // PML membership and compact aux index per direction
  const int *nabs = g.nabs;
  long px_ = -1, py_ = -1, pz_ = -1;
  if (i < nabs[0] || i >= g.ni - nabs[1]) {
    const int xa = (i < nabs[0]) ? i : i - (g.ni - nabs[1]) + g.xaoff;
    px_ = ((long)iz * g.nyi + iy) * g.nxa + xa;
  }
  if (j < nabs[2] || j >= g.nj - nabs[3]) {
    const int ya = (j < nabs[2]) ? j : j - (g.nj - nabs[3]) + nabs[2];
    py_ = ((long)iz * g.nya + ya) * g.px + ix;
  }
  if (k < nabs[4] || k >= g.nk - nabs[5]) {
    const int za = (k < nabs[4]) ? k : k - (g.nk - nabs[5]) + nabs[4];
    pz_ = ((long)za * g.nyi + iy) * g.px + ix;
  }
  float hax[9], hay[9], haz[9];
  if (px_ >= 0) {
    const float APDx = a.apd[0][ix], DBx = a.db[0][ix];
    const size_t as = g.astride[0];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const float av = a.ain[0][q * as + px_];
      hw[q] -= av / Bx;
      hax[q] = dxi[q] * DBx - APDx * av;
    }
    if (iz == g.top) {
      const float z1 = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz;
      const float z2 = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz;
      const float z3 = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz;
      const float f = DBx * Bx;
      hax[TXX] += f * (lam2mu * ztx * z1 + lambda * zty * z2 + lambda * ztz * z3);
      hax[TYY] += f * (lambda * ztx * z1 + lam2mu * zty * z2 + lambda * ztz * z3);
      hax[TZZ] += f * (lambda * ztx * z1 + lambda * zty * z2 + lam2mu * ztz * z3);
      hax[TXY] += f * (zty * z1 + ztx * z2) * miu;
      hax[TXZ] += f * (ztz * z1 + ztx * z3) * miu;
      hax[TYZ] += f * (ztz * z2 + zty * z3) * miu;
    }
  }
  if (py_ >= 0) {
    const float APDy = a.apd[1][iy], DBy = a.db[1][iy];
    const size_t as = g.astride[1];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const float av = a.ain[1][q * as + py_];
      hw[q] -= av / By;
      hay[q] = det[q] * DBy - APDy * av;
    }
    if (iz == g.top) {
      const float z1 = cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz;
      const float z2 = cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz;
      const float z3 = cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz;
      const float f = DBy * By;
      hay[TXX] += f * (lam2mu * ztx * z1 + lambda * zty * z2 + lambda * ztz * z3);
      hay[TYY] += f * (lambda * ztx * z1 + lam2mu * zty * z2 + lambda * ztz * z3);
      hay[TZZ] += f * (lambda * ztx * z1 + lambda * zty * z2 + lam2mu * ztz * z3);
      hay[TXY] += f * (zty * z1 + ztx * z2) * miu;
      hay[TXZ] += f * (ztz * z1 + ztx * z3) * miu;
      hay[TYZ] += f * (ztz * z2 + zty * z3) * miu;
    }
  }
  if (pz_ >= 0) {
    const float APDz = a.apd[2][iz], DBz = a.db[2][iz];
    const size_t as = g.astride[2];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const float av = a.ain[2][q * as + pz_];
      hw[q] -= av / Bz;
      haz[q] = dzt[q] * DBz - APDz * av;
    }
  }

  // ---- traction image for the velocities of the top 3 layers (CalTIMGmix) ----
  if (iz >= g.top - 2) {
    const int s = g.top - iz;  // the surface is s layers above this cell
    const float rhojac = a.flat ? irho : irho / a.jac[c];
    const int TC[3][3] = {{TXX, TXY, TXZ}, {TXY, TYY, TYZ}, {TXZ, TYZ, TZZ}};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float *T1 = in + TC[q][0] * fs, *T2 = in + TC[q][1] * fs, *T3 = in + TC[q][2] * fs;
      float vx[7], vy[7], vz[7];
#pragma unroll
      for (int n = 0; n < 7; ++n) {
        const long gx = c + (n - 3) * sx, gy = c + (n - 3) * sy, gz = c + (n - 3) * sz;
        if (a.flat) {
          vx[n] = T1[gx];
          vy[n] = T2[gy];
          vz[n] = T3[gz];
        } else {
          vx[n] = a.jac[gx] * T1[gx];
          vy[n] = a.jac[gy] * T2[gy];
          vz[n] = a.jac[gz] * (a.zx[gz] * T1[gz] + a.zy[gz] * T2[gz] + a.zz[gz] * T3[gz]);
        }
      }
#pragma unroll
      for (int p = 1; p <= LFD; ++p)
        if (p <= LFD - s) vz[3 + s + p] = -vz[3 + s - p];
      vz[3 + s] = 0.f;
      const float DxT = rhojac * strf7(vx, a.X, rx);
      const float DyT = rhojac * strf7(vy, a.Y, ry);
      const float DzT = rhojac * strf7(vz, a.Z, rz);
      float hv = DxT / Bx + DyT / By + DzT;
      if (px_ >= 0) {
        const float av = a.ain[0][q * g.astride[0] + px_];
        hv -= av / Bx;
        hax[q] = a.db[0][ix] * DxT - a.apd[0][ix] * av;
      }
      if (py_ >= 0) {
        const float av = a.ain[1][q * g.astride[1] + py_];
        hv -= av / By;
        hay[q] = a.db[1][iy] * DyT - a.apd[1][iy] * av;
      }
      hw[q] = hv;
    }
  }

  // ---- RK update (Iteration*) ----
  float *out = static_cast<float *>(a.out), *tw = static_cast<float *>(a.tw);
  const float *fw = static_cast<const float *>(a.fw);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const size_t o = q * fs + c;
    float twv = (RK == 0) ? 0.f : tw[o];
    const float fwv = (RK == 0) ? in[o] : ((RK < 3) ? fw[o] : 0.f);
    float outv;
    rk_update<RK>(hw[q], fwv, outv, twv, a.adt, a.bdt);
    out[o] = outv;
    if (RK < 3) tw[o] = twv;
  }
  // aux: ain is FA (rk 0) or A, afw is FA, aout is A (rk < 3) or FA (rk 3);
  // every aux value is read and written only by the thread of its own cell
  auto aux_update = [&](int d, long p, const float *hh) {
    const size_t as = g.astride[d];
    float *aout = a.aout[d], *ta = a.ta[d];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const size_t o = q * as + p;
      if (RK == 0) {
        const float f = a.ain[d][o];
        aout[o] = f + a.adt * hh[q];
        ta[o] = f + a.bdt * hh[q];
      } else if (RK < 3) {
        aout[o] = a.afw[d][o] + a.adt * hh[q];
        ta[o] = ta[o] + a.bdt * hh[q];
      } else {
        aout[o] = ta[o] + a.bdt * hh[q];
      }
    }
  };
  if (px_ >= 0) aux_update(0, px_, hax);
  if (py_ >= 0) aux_update(1, py_, hay);
  if (pz_ >= 0) aux_update(2, pz_, haz);
}

}  // namespace

void launch_stage_simple(const StageArgs &a, void *stream) {
  dim3 block(32, 4, 1);
  dim3 grid((a.g.ni + 31) / 32, (a.g.nj + 3) / 4, a.g.nk);
  cudaStream_t s = (cudaStream_t)stream;
  switch (a.rk) {
    case 0: stage_simple_kernel<0><<<grid, block, 0, s>>>(a); break;
    case 1: stage_simple_kernel<1><<<grid, block, 0, s>>>(a); break;
    case 2: stage_simple_kernel<2><<<grid, block, 0, s>>>(a); break;
    default: stage_simple_kernel<3><<<grid, block, 0, s>>>(a); break;
  }
}

}  // namespace cgfd
