// timg.cu -- traction-image velocity update of the top 3 layers, for the
// fused stage kernels (which skip those cells).
//
// Same arithmetic as the reference's CalTIMGmix (src/calculate.cu:5668-5897):
// on the 3 layers below and at the free surface, dV/dt comes from the
// conservative momentum equation
//     dV/dt = (1 / (rho J)) [ d_xi(J sigma.grad xi) + d_eta(J sigma.grad eta)
//                             + d_zeta(J sigma.grad zeta) ],
// with J sigma.grad zeta (the traction on zeta planes) set to zero on the
// surface layer and mirrored oddly above it.  Under SimpleCar grad xi and
// grad eta are the unit x and y vectors.  The x/y CFS-PML auxiliaries of V
// take their traction-image form; the RK update (Iteration*) is applied here
// for those cells.  A plain per-cell kernel: it touches 3 planes only.
#include "cgfd_internal.cuh"

#include <cuda_runtime.h>

namespace cgfd {
namespace {

__device__ __forceinline__ float drp5(float m1, float c0, float p1, float p2, float p3, float r) {
  return (CGFD_DA_1 * m1 + CGFD_DA0 * c0 + CGFD_DA1 * p1 + CGFD_DA2 * p2 + CGFD_DA3 * p3) * r;
}

// one cell (i, j) of layer iz
template <typename T>
__device__ __forceinline__ void timg_cell(const StageArgs &a, int i, int j, int iz) {
  using E = Elem<T>;
  const Geom &g = a.g;
  if (i >= g.ni || j >= g.nj) return;
  const int ix = i + XO, iy = j + LFD;
  const long c = (long)gidx(g, ix, iy, iz);
  const size_t fs = g.fstride;
  const long sy = g.px, sz = (long)g.plane;
  const int s = g.top - iz;  // the surface lies s layers above
  const float rx = a.X / a.h, ry = a.Y / a.h, rz = a.Z / a.h;
  const float irho = a.irho[c];
  const float rhojac = a.flat ? irho : irho / a.jac[c];
  const float iBx = 1.f / a.b[0][ix], iBy = 1.f / a.b[1][iy];
  const bool xpml = i < g.nabs[0] || i >= g.ni - g.nabs[1];
  const bool ypml = j < g.nabs[2] || j >= g.nj - g.nabs[3];
  const int xa = (i < g.nabs[0]) ? i : i - (g.ni - g.nabs[1]) + g.xaoff;
  const int ya = (j < g.nabs[2]) ? j : j - (g.nj - g.nabs[3]) + g.nabs[2];
  const size_t px = ((size_t)iz * g.nyi + iy) * g.nxa + xa;
  const size_t py = ((size_t)iz * g.nya + ya) * g.px + ix;
  const int kind = a.rk == 0 ? 0 : (a.rk < 3 ? 1 : 2);
  constexpr int TC[3][3] = {{TXX, TXY, TXZ}, {TXY, TYY, TYZ}, {TXZ, TYZ, TZZ}};
  const T *in = static_cast<const T *>(a.in);
  const T *fw = static_cast<const T *>(a.fw);
  T *out = static_cast<T *>(a.out), *tw = static_cast<T *>(a.tw);

#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const T *T1 = in + TC[q][0] * fs, *T2 = in + TC[q][1] * fs, *T3 = in + TC[q][2] * fs;
    // stored units to values (exact powers of two)
    const float s1 = a.sc[TC[q][0]], s2 = a.sc[TC[q][1]], s3 = a.sc[TC[q][2]];
    float vx[5], vy[5], vz[7];
#pragma unroll
    for (int d = -1; d <= 3; ++d) {
      const long gx = c + a.X * d, gy = c + a.Y * d * sy;
      vx[d + 1] = (a.flat ? 1.f : a.jac[gx]) * (E::ld(T1 + gx) * s1);
      vy[d + 1] = (a.flat ? 1.f : a.jac[gy]) * (E::ld(T2 + gy) * s2);
    }
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      const long gz = c + (n - 3) * sz;
      const float t1 = E::ld(T1 + gz) * s1, t2 = E::ld(T2 + gz) * s2, t3 = E::ld(T3 + gz) * s3;
      vz[n] = a.flat ? t3 : a.jac[gz] * (a.zx[gz] * t1 + a.zy[gz] * t2 + a.zz[gz] * t3);
    }
    if (s == 0) {
      vz[3] = 0.f; vz[4] = -vz[2]; vz[5] = -vz[1]; vz[6] = -vz[0];
    } else if (s == 1) {
      vz[4] = 0.f; vz[5] = -vz[3]; vz[6] = -vz[2];
    } else {
      vz[5] = 0.f; vz[6] = -vz[4];
    }
    const float DxT = rhojac * drp5(vx[0], vx[1], vx[2], vx[3], vx[4], rx);
    const float DyT = rhojac * drp5(vy[0], vy[1], vy[2], vy[3], vy[4], ry);
    const float DzT = a.Z > 0 ? rhojac * drp5(vz[2], vz[3], vz[4], vz[5], vz[6], rz)
                              : rhojac * drp5(vz[4], vz[3], vz[2], vz[1], vz[0], rz);
    float hv = DxT * iBx + DyT * iBy + DzT;
    // auxiliaries: X then Y, each read before it is written (own cell only)
    // under tW elision the first stage writes no tW and the second rebuilds
    // it (StageArgs::tw_skip)
    const bool rebuild = a.tw_skip && a.rk == 1;
    auto aux = [&](int d, size_t p, float h) {
      const size_t o = q * g.astride[d] + p;
      const float ai = a.ain[d][o];
      if (kind == 0) {
        a.aout[d][o] = ai + a.adt * h;
        a.ta[d][o] = ai + a.bdt * h;
      } else if (kind == 1) {
        const float f = a.afw[d][o], t = a.ta[d][o];
        a.aout[d][o] = f + a.adt * h;
        a.ta[d][o] = t + a.bdt * h;
      } else {
        a.aout[d][o] = a.ta[d][o] + a.bdt * h;
      }
    };
    float hax = 0.f, hay = 0.f;
    if (xpml) {
      const float ai = a.ain[0][q * g.astride[0] + px];
      hv -= ai * iBx;
      hax = a.db[0][ix] * DxT - a.apd[0][ix] * ai;
    }
    if (ypml) {
      const float ai = a.ain[1][q * g.astride[1] + py];
      hv -= ai * iBy;
      hay = a.db[1][iy] * DyT - a.apd[1][iy] * ai;
    }
    if (xpml) aux(0, px, hax);
    if (ypml) aux(1, py, hay);
    // RK update in stored units (every set of a component shares its scale)
    const size_t o = (size_t)(VX + q) * fs + c;
    const float adt = a.adt * a.isc[VX + q], bdt = a.bdt * a.isc[VX + q];
    // 16-bit storage keeps tW as tW - FW (the paired kernels' form)
    constexpr bool D = sizeof(T) != 4;
    if (kind == 0) {
      const float u0 = E::ld(in + o);
      E::st(out + o, u0 + adt * hv);
      if (!a.tw_skip) E::st(tw + o, D ? bdt * hv : u0 + bdt * hv);
    } else if (kind == 1) {
      const float u0 = E::ld(fw + o);
      float u1;
      if (rebuild) u1 = D ? a.rtw * (E::ld(in + o) - u0) : u0 + a.rtw * (E::ld(in + o) - u0);
      else u1 = E::ld(tw + o);
      E::st(out + o, u0 + adt * hv);
      E::st(tw + o, u1 + bdt * hv);
    } else {
      const float t = D ? E::ld(fw + o) + E::ld(tw + o) : E::ld(tw + o);
      E::st(out + o, t + bdt * hv);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(128) timg_kernel(StageArgs a) {
  timg_cell<T>(a, blockIdx.x * 32 + threadIdx.x, blockIdx.y * 4 + threadIdx.y,
               a.g.top - 2 + blockIdx.z);
}

// n models: blockIdx.z = model * 3 + layer; the grid covers the largest model
template <typename T>
__global__ void __launch_bounds__(128) timg_batch_kernel(const StageArgs *args) {
  const StageArgs &a = args[blockIdx.z / 3];
  timg_cell<T>(a, blockIdx.x * 32 + threadIdx.x, blockIdx.y * 4 + threadIdx.y,
               a.g.top - 2 + (int)(blockIdx.z % 3));
}

}  // namespace

void launch_timg_batch(const StageArgs *args, int n, int max_ni, int max_nj, int elem,
                       void *stream) {
  dim3 block(32, 4, 1);
  dim3 grid((max_ni + 31) / 32, (max_nj + 3) / 4, 3 * n);
  cudaStream_t s = (cudaStream_t)stream;
  if (elem == ELEM_F16) timg_batch_kernel<__half><<<grid, block, 0, s>>>(args);
  else if (elem == ELEM_BF16) timg_batch_kernel<__nv_bfloat16><<<grid, block, 0, s>>>(args);
  else timg_batch_kernel<float><<<grid, block, 0, s>>>(args);
}

void launch_timg(const StageArgs &a, void *stream) {
  dim3 block(32, 4, 1);
  dim3 grid((a.g.ni + 31) / 32, (a.g.nj + 3) / 4, 3);
  if (a.elem == ELEM_F16)
    timg_kernel<__half><<<grid, block, 0, (cudaStream_t)stream>>>(a);
  else if (a.elem == ELEM_BF16)
    timg_kernel<__nv_bfloat16><<<grid, block, 0, (cudaStream_t)stream>>>(a);
  else
    timg_kernel<float><<<grid, block, 0, (cudaStream_t)stream>>>(a);
}

}  // namespace cgfd
