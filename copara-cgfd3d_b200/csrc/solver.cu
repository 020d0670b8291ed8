// solver.cu -- C ABI (include/cgfd.h) of the B200 CGFD solver: device state,
// uploads with layout conversion, the per-step CUDA graphs, sources,
// receivers and diagnostics.
//
// Reference counterparts: class ChildProcs (src/typedata.h:114-217) and its
// methods in src/calculate.cu (ctor 107-1005, ParH2D 2050-2228, VelCoeff
// 1336-1353, RKite 1355-1600, wavesyn/abssyn 2956-3119, C2DPointPick/PWpick
// 2678-2830), driven by the step loop of src/simulation.cc:252-711.
#include "../../include/cgfd.h"
#include "abi_guard.h"
#include "cgfd_internal.cuh"
#include "ncwrite.h"
#include "nonfinite.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace cgfd;
using namespace cgfd::nf;

namespace {

// the last error of a call without a handle, per host thread (cgfd_last_error
// with NULL reads the calling thread's)
thread_local std::string g_last_create_error;

// RK4 coefficients (src/calculate.cu:12-13).
constexpr double RKA[3] = {0.5, 0.5, 1.0};
constexpr double RKB[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
// F/B direction triples per step%4 and stage (src/simulation.cc:264-641).
constexpr int DIRS[4][4][3] = {
    {{1, 1, 1}, {-1, -1, -1}, {1, 1, 1}, {-1, -1, -1}},
    {{1, 1, -1}, {-1, -1, 1}, {1, 1, -1}, {-1, -1, 1}},
    {{-1, -1, -1}, {1, 1, 1}, {-1, -1, -1}, {1, 1, 1}},
    {{-1, -1, 1}, {1, 1, -1}, {-1, -1, 1}, {1, 1, -1}}};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// ------------------------------ kernels -----------------------------------

// reference layout (i*ny+j)*nz+k  ->  internal layout (x fastest), stored
// as T in units of 1/isc
template <typename T>
__global__ void to_internal_kernel(const float *__restrict__ src, T *__restrict__ dst, Geom g,
                                   int nx, int ny, int nz, float isc) {
  const long n = (long)nx * ny * nz;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    const int k = (int)(q % nz);
    const long r = q / nz;
    const int j = (int)(r % ny);
    const int i = (int)(r / ny);
    Elem<T>::st(dst + gidx(g, i + XSH, j, k), src[q] * isc);
  }
}
template <typename T>
__global__ void to_reference_kernel(const T *__restrict__ src, float *__restrict__ dst, Geom g,
                                    int nx, int ny, int nz, float sc) {
  const long n = (long)nx * ny * nz;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    const int k = (int)(q % nz);
    const long r = q / nz;
    const int j = (int)(r % ny);
    const int i = (int)(r / ny);
    dst[q] = Elem<T>::ld(src + gidx(g, i + XSH, j, k)) * sc;
  }
}

// Point sources (LoadMoment/LoadForce, src/calculate.cu:6130-6255), applied
// to the stage output; one thread walks the list so that repeated cells add
// up in a fixed order.
// W_out += adt*S, tW += bdt*S in stored units of the component (the last
// stage: W_out += bdt*S)
template <typename T>
__device__ __forceinline__ void add_stage_term(const SourceArgs &s, int comp, size_t o, float S) {
  using E = Elem<T>;
  T *out = static_cast<T *>(s.out), *tw = static_cast<T *>(s.tw);
  const float a = s.adt * s.isc[comp], b = s.bdt * s.isc[comp];
  if (s.rk == 3) {
    E::st(out + o, E::ld(out + o) + b * S);
  } else {
    E::st(out + o, E::ld(out + o) + a * S);
    // under tW elision the first stage's tW is rebuilt from W later, and
    // W already carries this source term
    if (!(s.tw_skip && s.rk == 0)) E::st(tw + o, E::ld(tw + o) + b * S);
  }
}
template <typename T>
__device__ void inject_sources_body(const SourceArgs &s) {
  const int t2 = (s.tindex >= 0) ? s.tindex : 2 * (*s.step) + s.tinc;
  const size_t fs = s.g.fstride;
  auto add = [&](int comp, size_t o, float S) { add_stage_term<T>(s, comp, o, S); };
  for (int q = 0; q < ((s.smooth & 1u) ? 0 : s.nmnt); ++q) {
    const float stf = s.mstf[(size_t)q * s.nstfm + t2];
    const int c = s.mcell[q];
    for (int m = 0; m < 6; ++m)
      add(TXX + m, (size_t)(TXX + m) * fs + c, -s.mcoef[6 * q + m] * stf);
  }
  for (int q = 0; q < ((s.smooth & 2u) ? 0 : s.nfrc); ++q) {
    const float stf = s.fstf[(size_t)q * s.nstff + t2];
    const int c = s.fcell[q];
    for (int m = 0; m < 3; ++m) add(VX + m, (size_t)(VX + m) * fs + c, stf * s.fcoef[3 * q + m]);
  }
}
// tW elision, single-stage driving: after a first stage run alone, tW (valid
// cells) is written as the reference's first stage leaves it,
// tW = FW + r * (W - FW), so the state between stages matches the
// reference's; the next stage rebuilds it the same way anyway.  16-bit
// storage keeps tW as its difference from FW (the stage kernels' form):
// r * (W - FW).
template <typename T>
__global__ void rebuild_tw_kernel(Geom g, const T *fw, const T *w, T *tw, float r) {
  using E = Elem<T>;
  constexpr bool D = sizeof(T) != 4;
  const long n = (long)g.ni * g.nj * g.nk;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
       t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.ni), j = (int)(t / g.ni % g.nj), k = (int)(t / ((long)g.ni * g.nj));
    const size_t o = gidx(g, i + XO, j + LFD, k + LFD);
    for (int c = 0; c < NCOMP; ++c) {
      const size_t q = (size_t)c * g.fstride + o;
      const float f = E::ld(fw + q);
      E::st(tw + q, D ? r * (E::ld(w + q) - f) : f + r * (E::ld(w + q) - f));
    }
  }
}
template <typename T>
__global__ void inject_sources_kernel(SourceArgs s) {
  if (threadIdx.x == 0 && blockIdx.x == 0) inject_sources_body<T>(s);
}
// a batch of models (one storage type): block b injects model b's sources
template <typename T>
__global__ void inject_sources_batch_kernel(const SourceArgs *sa) {
  if (threadIdx.x == 0) inject_sources_body<T>(sa[blockIdx.x]);
}
// Focal points (LoadRmom without SrcSmooth, src/calculate.cu:6257-6319):
// each adds -M(t) / (h^3 J) to its cell's stress RHS; M(t) as the
// reference's ExtractValue (src/calculate.cu:2586-2613) computes it, in
// single precision as there: linear between the samples PL and PR =
// PL + 1, PR = PL when t lies within 1e-5 s of a sample, zero outside
// [0, dt*(n-1)] (indices are also clamped to the series).  Points may share
// a cell, hence atomic additions.
__device__ __forceinline__ float focal_value(const float *stf, int n, float DT, float time) {
  const float Tend = DT * (float)(n - 1);
  if (time > Tend || time < 0.f) return 0.f;
  int PL = (int)(time / DT);
  const bool on = (double)fabsf(time - DT * floorf(time / DT)) < 1e-5;
  int PR = on ? PL : PL + 1;
  PL = PL < n - 1 ? PL : n - 1;
  PR = PR < n - 1 ? PR : n - 1;
  return stf[PL] + (stf[PR] - stf[PL]) * ((time - DT * (float)PL) / DT);
}
__device__ __forceinline__ void atomic_add_elem(float *p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_elem(__half *p, float v) {
  atomicAdd(p, __float2half_rn(v));
}
__device__ __forceinline__ void atomic_add_elem(__nv_bfloat16 *p, float v) {
  atomicAdd(p, __float2bfloat16_rn(v));
}
template <typename T>
__device__ void inject_focal_body(const SourceArgs &s, int t0, int tstride) {
  // the stage's time (src/calculate.cu:1422): (currT + tinc/2) * stept
  const int currT = (s.tindex >= 0) ? (s.tindex - s.tinc) / 2 : *s.step;
  const float time = (float)(((double)currT + s.tinc * 0.5) * (double)s.dt);
  const float h3 = s.h * s.h * s.h;
  const size_t fs = s.g.fstride;
  T *out = static_cast<T *>(s.out), *tw = static_cast<T *>(s.tw);
  const bool to_tw = s.rk != 3 && !(s.tw_skip && s.rk == 0);
  if (s.smooth & 4u) return;
  for (int q = t0; q < s.nfoc; q += tstride) {
    const int c = s.foccell[q];
    const float A = 1.f / (h3 * s.jac[c]);
    for (int m = 0; m < 6; ++m) {
      const float M = focal_value(s.focmom + ((size_t)m * s.nfoc + q) * s.fnt, s.fnt, s.fdt, time);
      const float S = -M * A;
      const int comp = TXX + m;
      const size_t o = (size_t)comp * fs + c;
      const float a = s.adt * s.isc[comp], b = s.bdt * s.isc[comp];
      atomic_add_elem(out + o, (s.rk == 3 ? b : a) * S);
      if (to_tw) atomic_add_elem(tw + o, b * S);
    }
  }
}
template <typename T>
__global__ void inject_focal_kernel(SourceArgs s) {
  inject_focal_body<T>(s, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
// a batch of models (one storage type): blockIdx.y = model
template <typename T>
__global__ void inject_focal_batch_kernel(const SourceArgs *sa) {
  inject_focal_body<T>(sa[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x,
                       gridDim.x * blockDim.x);
}
// Smoothed sources (the SrcSmooth forms of LoadMoment, LoadForce and
// LoadRmom, src/calculate.cu:6147-6175, 6210-6232, 6275-6296): one thread
// per node of the spread list sums its entries in list order, then adds
// the sum once per component, so the result does not depend on thread
// timing.  Entry coefficients: moments 6 x w / (h^3 J), forces 3 x
// w / (h^3 J rho) (x2 on the surface), focal points w / (h^3 J) in [0].
template <typename T>
__device__ void inject_spread_body(const SourceArgs &s, int u0, int ustride) {
  const int t2 = (s.tindex >= 0) ? s.tindex : 2 * (*s.step) + s.tinc;
  const int currT = (s.tindex >= 0) ? (s.tindex - s.tinc) / 2 : *s.step;
  const float time = (float)(((double)currT + s.tinc * 0.5) * (double)s.dt);
  const size_t fs = s.g.fstride;
  for (int u = u0; u < s.nsp; u += ustride) {
    float S[NCOMP] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    bool vel = false, str = false;
    for (int e = s.spoff[u]; e < s.spoff[u + 1]; ++e) {
      const int r = s.sprow[e], kind = r >> 28, q = r & 0x0fffffff;
      const float *c = s.spcoef + (size_t)6 * e;
      if (kind == 0) {
        const float stf = s.mstf[(size_t)q * s.nstfm + t2];
        for (int m = 0; m < 6; ++m) S[TXX + m] -= c[m] * stf;
        str = true;
      } else if (kind == 1) {
        const float stf = s.fstf[(size_t)q * s.nstff + t2];
        for (int m = 0; m < 3; ++m) S[VX + m] += c[m] * stf;
        vel = true;
      } else {
        for (int m = 0; m < 6; ++m)
          S[TXX + m] -= c[0] * focal_value(s.focmom + ((size_t)m * s.nfoc + q) * s.fnt, s.fnt,
                                           s.fdt, time);
        str = true;
      }
    }
    const size_t cell = (size_t)s.spcell[u];
    if (vel)
      for (int m = 0; m < 3; ++m) add_stage_term<T>(s, VX + m, (size_t)(VX + m) * fs + cell, S[VX + m]);
    if (str)
      for (int m = 0; m < 6; ++m)
        add_stage_term<T>(s, TXX + m, (size_t)(TXX + m) * fs + cell, S[TXX + m]);
  }
}
template <typename T>
__global__ void inject_spread_kernel(SourceArgs s) {
  inject_spread_body<T>(s, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
// a batch of models (one storage type): blockIdx.y = model
template <typename T>
__global__ void inject_spread_batch_kernel(const SourceArgs *sa) {
  inject_spread_body<T>(sa[blockIdx.y], blockIdx.x * blockDim.x + threadIdx.x,
                        gridDim.x * blockDim.x);
}
int spread_blocks(int nsp) { return nsp <= 0 ? 1 : ((nsp + 127) / 128 < 296 ? (nsp + 127) / 128 : 296); }
void launch_spread(const SourceArgs &s, cudaStream_t st) {
  const int nb = spread_blocks(s.nsp);
  if (s.elem == ELEM_F16) inject_spread_kernel<__half><<<nb, 128, 0, st>>>(s);
  else if (s.elem == ELEM_BF16) inject_spread_kernel<__nv_bfloat16><<<nb, 128, 0, st>>>(s);
  else inject_spread_kernel<float><<<nb, 128, 0, st>>>(s);
}
int focal_blocks(int nfoc) { return nfoc <= 0 ? 1 : ((nfoc + 127) / 128 < 296 ? (nfoc + 127) / 128 : 296); }
void launch_focal(const SourceArgs &s, cudaStream_t st) {
  const int nb = focal_blocks(s.nfoc);
  if (s.elem == ELEM_F16) inject_focal_kernel<__half><<<nb, 128, 0, st>>>(s);
  else if (s.elem == ELEM_BF16) inject_focal_kernel<__nv_bfloat16><<<nb, 128, 0, st>>>(s);
  else inject_focal_kernel<float><<<nb, 128, 0, st>>>(s);
}

void launch_sources(const SourceArgs &s, cudaStream_t st) {
  if (s.elem == ELEM_F16) inject_sources_kernel<__half><<<1, 32, 0, st>>>(s);
  else if (s.elem == ELEM_BF16) inject_sources_kernel<__nv_bfloat16><<<1, 32, 0, st>>>(s);
  else inject_sources_kernel<float><<<1, 32, 0, st>>>(s);
}

// Receiver recording (PWpick, src/calculate.cu:2780-2830) from FW after a
// step, into seis[(c*nrecv + r)*nt + t]; then advances the step counter.
template <typename T>
__device__ void record_body(const T *__restrict__ fw, size_t fstride,
                            const int *__restrict__ cells, int nrecv, int nt,
                            float *__restrict__ seis, int *step, const ScaleSet &s) {
  const int t = *step;
  for (int q = threadIdx.x; q < 9 * nrecv; q += blockDim.x) {
    const int c = q / nrecv, r = q % nrecv;
    if (t < nt)
      seis[((size_t)c * nrecv + r) * nt + t] =
          Elem<T>::ld(fw + (size_t)c * fstride + cells[r]) * s.sc[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) *step = t + 1;
}
template <typename T>
__global__ void record_kernel(const T *__restrict__ fw, size_t fstride,
                              const int *__restrict__ cells, int nrecv, int nt,
                              float *__restrict__ seis, int *step, ScaleSet s) {
  record_body<T>(fw, fstride, cells, nrecv, nt, seis, step, s);
}
// receiver record of one model of a batch (storage type of the batch)
struct RecordArgs {
  const void *fw;
  size_t fstride;
  const int *cells;
  int nrecv, nt;
  float *seis;
  int *step;
  ScaleSet s;
};
template <typename T>
__global__ void record_batch_kernel(const RecordArgs *ra) {
  const RecordArgs &r = ra[blockIdx.x];
  record_body<T>(static_cast<const T *>(r.fw), r.fstride, r.cells, r.nrecv, r.nt, r.seis, r.step,
                 r.s);
}

// multiplies component comp of the four field sets by factor (a power of two:
// exact unless it leaves the storage type's range)
template <typename T>
__global__ void rescale_kernel(T *sets, size_t fstride, int comp, float factor) {
  const size_t n = fstride;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x)
    for (int s = 0; s < 4; ++s) {
      T *p = sets + ((size_t)s * NCOMP + comp) * fstride + q;
      Elem<T>::st(p, Elem<T>::ld(p) * factor);
    }
}

// Peak ground velocity (IterationFinalPV, src/calculate.cu:6736-6851): after
// a step, max |V| per component over time at each surface cell of FW.
template <typename T>
__global__ void pgv_kernel(const T *__restrict__ fw, Geom g, float *__restrict__ pgv, float s0,
                           float s1, float s2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= g.ni || j >= g.nj) return;
  const size_t m = (size_t)(j + LFD) * g.px + i + XO;
  const size_t c = (size_t)g.top * g.plane + m;
  const float sc[3] = {s0, s1, s2};
  for (int q = 0; q < 3; ++q) {
    const float v = fabsf(Elem<T>::ld(fw + (size_t)q * g.fstride + c) * sc[q]);
    float *p = pgv + (size_t)q * g.plane + m;
    *p = fmaxf(*p, v);
  }
}

// Sub-volume of a field set (SWpick, src/calculate.cu:2230-2493): components
// in mask order, then i, j, k with k fastest, from reference indices
// start + n*stride.
template <typename T>
__global__ void snapshot_kernel(const T *__restrict__ set, Geom g, int mask, int3 st, int3 cnt,
                                int3 sd, ScaleSet s, float *__restrict__ out) {
  const long per = (long)cnt.x * cnt.y * cnt.z;
  int slot = 0;
  for (int c = 0; c < NCOMP; ++c) {
    if (!(mask & (1 << c))) continue;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < per;
         q += (long)gridDim.x * blockDim.x) {
      const int k = (int)(q % cnt.z), j = (int)((q / cnt.z) % cnt.y), i = (int)(q / cnt.z / cnt.y);
      const size_t o = (size_t)c * g.fstride +
                       gidx(g, st.x + i * sd.x + XSH, st.y + j * sd.y, st.z + k * sd.z);
      out[slot * per + q] = Elem<T>::ld(set + o) * s.sc[c];
    }
    ++slot;
  }
}

}  // namespace

struct cgfd_solver {
  cgfd_desc d{};
  Geom g{};
  cudaStream_t st = nullptr;
  // traction image and stress part beside the velocity part
  SideStream side{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // host-to-device upload staging: the copy events of the two pinned chunks
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  std::string err;
  void *state = nullptr;   // 4 sets of 9 components: FW, Wa, Wb, tW
  void *set[4] = {nullptr, nullptr, nullptr, nullptr};
  int elem = ELEM_F32;     // storage element type of the sets
  int sexp[NCOMP] = {};    // per-component scale exponents: stored = value * 2^-sexp
  bool user_scales = false;
  int wcur = 0;            // set that holds "W" (last stage output)
  float *media = nullptr;  // lam2mu, mu, irho
  float *metric = nullptr; // zeta_x, zeta_y, zeta_z, jac
  float *zzp = nullptr;    // per plane: uniform zeta_z below ConIndex
  int zu_end = 0;          // planes iz < zu_end have one (zzp)
  float *pml = nullptr;    // apd x y z, b x y z, db x y z
  float *pmlp[9] = {};
  float *aux[3] = {nullptr, nullptr, nullptr};  // per direction: FA, A, tA sets
  float *matv = nullptr;
  bool flat = false, have_metric = false, have_media = false, have_pml = false;
  bool prepared = false;
  // host copies needed by the FP64 free-surface matrices
  std::vector<double> top_zeta;            // 3 * nx * ny (surface layer)
  std::vector<double> top_alpha, top_beta, top_rho;  // nx * ny
  std::vector<double> hb[3];               // B profiles
  // sources
  int nmnt = 0, nfrc = 0, nstfm = 0, nstff = 0;
  std::vector<int> mloc, floc;
  std::vector<float> m6, f3;
  std::vector<float> hmstf, hfstf;  // host copies of the source time functions
  int *d_mcell = nullptr, *d_fcell = nullptr;
  float *d_mcoef = nullptr, *d_fcoef = nullptr, *d_mstf = nullptr, *d_fstf = nullptr;
  // focal (finite-fault) points: cells and moment series [6][nfoc][fnt]
  int nfoc = 0, fnt = 0;
  double fdt = 0;
  std::vector<int> focloc;
  std::vector<float> hfocmom;
  int *d_foccell = nullptr;
  float *d_focmom = nullptr;
  // source smoothing weights per kind (moments, forces, focal points),
  // [n][7][7][7]; the spread list by node that prepare builds from them
  std::vector<double> smw[3];
  int sp_n = 0;
  int *d_sp_cell = nullptr, *d_sp_off = nullptr, *d_sp_row = nullptr;
  float *d_sp_coef = nullptr;
  // receivers
  int nrecv = 0;
  int *d_rcell = nullptr;
  float *d_seis = nullptr;
  int *d_step = nullptr;
  int steps = 0;
  unsigned long long *d_partials = nullptr;  // non-finite count scratch
  int nf_blocks = 0;
  // graphs (one per step%4 pattern)
  cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
  bool graphs_ok = false;
  float *d_pgv = nullptr;  // peak ground velocity, [3][plane] at the surface (optional)
  // learned absorbing layer (optional): cells {internal index, normal
  // offset, 0, 0}, their reference indices, FP16 weights, 9 x n scratch
  int mlp_n = 0;
  int4 *d_mlp_cells = nullptr;
  std::vector<int> mlp_ijk;
  void *d_mlp_w = nullptr;
  float *d_mlp_delta = nullptr;
  float *d_mlp_gain = nullptr;  // [width][9]
  int mlp_width = 0;
  // fused kernels: tensor maps and launch shape; device error flag (bounded
  // waits that expired, alignment self-check)
  void *plan = nullptr;
  int *d_err = nullptr;
  bool plain_interior = true;
};

void cgfd::set_global_error(const char *msg) { g_last_create_error = msg; }

namespace {

// "fn: host allocation or thread failure (what)" for the exception being
// handled (called from inside a catch handler only)
void exception_text(const char *fn, char *buf, size_t len) noexcept {
  const char *what = "unknown C++ exception";
  try {
    throw;
  } catch (const std::exception &e) {
    what = e.what();
  } catch (...) {
  }
  std::snprintf(buf, len, "%s: host allocation or thread failure (%s)", fn, what);
}

}  // namespace

int cgfd::abi_exception(const cgfd_solver *h, const char *fn) noexcept {
  char buf[320];
  exception_text(fn, buf, sizeof(buf));
  try {
    if (h) const_cast<cgfd_solver *>(h)->err = buf;
    else g_last_create_error = buf;
  } catch (...) {
  }
  return CGFD_ERR_NOMEM;
}

namespace {

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int cuda_fail(cgfd_solver *h, cudaError_t e, const char *what) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
  if (h) h->err = buf; else g_last_create_error = buf;
  return CGFD_ERR_CUDA;
}
int arg_fail(cgfd_solver *h, const char *what) {
  if (h) h->err = what; else g_last_create_error = what;
  return CGFD_ERR_ARG;
}

#define CK(h, call)                                         \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
  } while (0)

void free_all(cgfd_solver *h) {
  if (h->plan) {
    if (h->d.kernel == CGFD_KERNEL_FUSED) pair_destroy_plan(h->plan);
    else fused_destroy_plan(h->plan);
    h->plan = nullptr;
  }
  for (auto &gr : h->graph)
    if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; }
  void *ptrs[] = {h->state, h->media, h->metric, h->pml, h->aux[0], h->aux[1], h->aux[2],
                  h->matv, h->d_mcell, h->d_fcell, h->d_mcoef, h->d_fcoef, h->d_mstf,
                  h->d_fstf, h->d_rcell, h->d_seis, h->d_step, h->d_partials, h->d_err,
                  h->d_pgv, h->d_mlp_cells, h->d_mlp_w, h->d_mlp_delta, h->zzp,
                  h->d_foccell, h->d_focmom, h->d_sp_cell, h->d_sp_off, h->d_sp_row,
                  h->d_sp_coef};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (h->st) cudaStreamDestroy(h->st);
  for (int q = 0; q < 2; ++q)
    if (h->pin_ev[q]) cudaEventDestroy(h->pin_ev[q]);
  if (h->side.stream) cudaStreamDestroy((cudaStream_t)h->side.stream);
  if (h->side.fork) cudaEventDestroy((cudaEvent_t)h->side.fork);
  if (h->side.join) cudaEventDestroy((cudaEvent_t)h->side.join);
  if (h->side.stream2) cudaStreamDestroy((cudaStream_t)h->side.stream2);
  if (h->side.fork2) cudaEventDestroy((cudaEvent_t)h->side.fork2);
  if (h->side.join2) cudaEventDestroy((cudaEvent_t)h->side.join2);
}

long ref_n(const cgfd_solver *h) {
  return (long)(h->d.ni + 6) * (h->d.nj + 6) * (h->d.nk + 6);
}

// host float array (reference layout) -> internal array at dst, stored as
// element type elem in units of 1/isc
int upload_ref(cgfd_solver *h, const float *host, void *dst, int elem = ELEM_F32,
               float isc = 1.f) {
  const long n = ref_n(h);
  float *tmp = nullptr;
  CK(h, cudaMalloc(&tmp, n * sizeof(float)));
  cudaError_t e = cudaMemcpyAsync(tmp, host, n * sizeof(float), cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) {
    const int nx = h->d.ni + 6, ny = h->d.nj + 6, nz = h->d.nk + 6;
    if (elem == ELEM_F16)
      to_internal_kernel<<<592, 256, 0, h->st>>>(tmp, (__half *)dst, h->g, nx, ny, nz, isc);
    else if (elem == ELEM_BF16)
      to_internal_kernel<<<592, 256, 0, h->st>>>(tmp, (__nv_bfloat16 *)dst, h->g, nx, ny, nz,
                                                  isc);
    else
      to_internal_kernel<<<592, 256, 0, h->st>>>(tmp, (float *)dst, h->g, nx, ny, nz, isc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(h, e, "upload");
  return CGFD_OK;
}

// a loop over [0, n) split over up to 16 host threads (serial when small)
template <class F>
void par_for(long n, F &&f) {
  unsigned nt = std::thread::hardware_concurrency();
  nt = nt ? (nt < 16u ? nt : 16u) : 4u;
  if (n < (1L << 18) || nt < 2) {
    f(0L, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (unsigned t = 0; t < nt; ++t) {
    const long b = n * (long)t / nt, e = n * (long)(t + 1) / nt;
    th.emplace_back([&f, b, e] { f(b, e); });
  }
  for (auto &x : th) x.join();
}

// Uploads `count` reference-layout arrays of ref_n floats into the internal
// layout of dst[a] (FP32): fill(a, b, e, out) writes elements [b, e) of array
// a (converted as the caller wants) to out[0 .. e-b).  Chunks pass through two
// pinned host buffers, each filled on host threads while the other's copy
// runs, into one device staging array, converted on the device per array.
// The two pinned buffers are one pool for the process (portable to every
// device, allocated at the first upload and kept until exit: page-locking
// 128 MB costs about a tenth of a second, which every new solver would pay
// again), used by one upload at a time.
constexpr long PIN_CHUNK = 16L << 20;  // floats per pinned buffer (64 MB)
std::mutex g_pin_mutex;
float *g_pin[2] = {nullptr, nullptr};
template <class Fill>
int upload_fields(cgfd_solver *h, int count, Fill &&fill, float *const *dst) {
  const long n = ref_n(h);
  std::lock_guard<std::mutex> lock(g_pin_mutex);
  for (int q = 0; q < 2; ++q) {
    if (!g_pin[q])
      CK(h, cudaHostAlloc((void **)&g_pin[q], PIN_CHUNK * sizeof(float), cudaHostAllocPortable));
    if (!h->pin_ev[q]) CK(h, cudaEventCreateWithFlags(&h->pin_ev[q], cudaEventDisableTiming));
  }
  float *tmp = nullptr;
  CK(h, cudaMalloc(&tmp, n * sizeof(float)));
  const int nx = h->d.ni + 6, ny = h->d.nj + 6, nz = h->d.nk + 6;
  cudaError_t e = cudaSuccess;
  int c = 0;
  for (int a = 0; a < count && e == cudaSuccess; ++a) {
    for (long b = 0; b < n && e == cudaSuccess; b += PIN_CHUNK, ++c) {
      const long end = b + PIN_CHUNK < n ? b + PIN_CHUNK : n;
      float *buf = g_pin[c & 1];
      e = cudaEventSynchronize(h->pin_ev[c & 1]);  // its previous copy is done
      if (e != cudaSuccess) break;
      par_for(end - b, [&](long x0, long x1) { fill(a, b + x0, b + x1, buf + x0); });
      e = cudaMemcpyAsync(tmp + b, buf, (end - b) * sizeof(float), cudaMemcpyHostToDevice, h->st);
      if (e == cudaSuccess) e = cudaEventRecord(h->pin_ev[c & 1], h->st);
    }
    if (e == cudaSuccess) {
      to_internal_kernel<<<592, 256, 0, h->st>>>(tmp, dst[a], h->g, nx, ny, nz, 1.f);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(h, e, "upload");
  return CGFD_OK;
}

int download_ref(cgfd_solver *h, const void *src, float *host, int elem = ELEM_F32,
                 float sc = 1.f) {
  const long n = ref_n(h);
  float *tmp = nullptr;
  CK(h, cudaMalloc(&tmp, n * sizeof(float)));
  const int nx = h->d.ni + 6, ny = h->d.nj + 6, nz = h->d.nk + 6;
  if (elem == ELEM_F16)
    to_reference_kernel<<<592, 256, 0, h->st>>>((const __half *)src, tmp, h->g, nx, ny, nz, sc);
  else if (elem == ELEM_BF16)
    to_reference_kernel<<<592, 256, 0, h->st>>>((const __nv_bfloat16 *)src, tmp, h->g, nx, ny,
                                                 nz, sc);
  else
    to_reference_kernel<<<592, 256, 0, h->st>>>((const float *)src, tmp, h->g, nx, ny, nz, sc);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host, tmp, n * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(h, e, "download");
  return CGFD_OK;
}

bool valid_loc(const cgfd_solver *h, const int *l) {
  return l[0] >= LFD && l[0] < h->d.ni + LFD && l[1] >= LFD && l[1] < h->d.nj + LFD &&
         l[2] >= LFD && l[2] < h->d.nk + LFD;
}
int cell_of(const cgfd_solver *h, const int *l) {
  return (int)gidx(h->g, l[0] + XSH, l[1], l[2]);
}

void invalidate(cgfd_solver *h) {
  h->prepared = false;
  h->graphs_ok = false;
}

// Free-surface velocity-gradient matrices in FP64 (VelPDcoeff under SimpleCar,
// src/calculate.cu:3320-3428): for each surface column, with e3 = grad zeta,
// A = C(e3,e3), B = C(e3,e1), C = C(e3,e2) of the isotropic stiffness, and
// matVx2Vz = -A^-1 B * Bz/Bx, matVy2Vz = -A^-1 C * Bz/By.  A is inverted by
// Gauss-Jordan without pivoting in the reference's order.
void surface_matrices(const cgfd_solver *h, std::vector<float> &out) {
  const int nx = h->d.ni + 6, ny = h->d.nj + 6, top = h->g.top;
  const size_t plane = h->g.plane;
  out.assign(18 * plane, 0.f);
  for (int i = LFD; i < h->d.ni + LFD; ++i)
    for (int j = LFD; j < h->d.nj + LFD; ++j) {
      const size_t t2 = (size_t)i * ny + j;
      const double rho = h->top_rho[t2], al = h->top_alpha[t2], be = h->top_beta[t2];
      const double mu = rho * be * be, l2m = rho * al * al, la = l2m - 2.0 * mu;
      const double e[3][3] = {{1, 0, 0}, {0, 1, 0},
                              {h->top_zeta[t2], h->top_zeta[(size_t)nx * ny + t2],
                               h->top_zeta[2 * (size_t)nx * ny + t2]}};
      // stiffness contraction K(p,q)[r][s] for row direction e_p and column e_q
      auto K = [&](const double *p, const double *q, double *m) {
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) {
            const double v = (r == s) ? (l2m * p[r] * q[r]) : (la * p[r] * q[s] + mu * p[s] * q[r]);
            m[r * 3 + s] = v;
          }
        // shear terms on the diagonal: mu*(sum over the other two axes)
        for (int r = 0; r < 3; ++r) {
          double sh = 0;
          for (int a = 0; a < 3; ++a)
            if (a != r) sh += p[a] * q[a];
          m[r * 3 + r] += mu * sh;
        }
      };
      double A[9], B[9], C[9];
      K(e[2], e[2], A);
      K(e[2], e[0], B);
      K(e[2], e[1], C);
      for (int r = 0; r < 3; ++r) {  // Gauss-Jordan, no pivoting
        double con = A[r * 3 + r];
        A[r * 3 + r] = 1;
        for (int s = 0; s < 3; ++s) A[r * 3 + s] /= con;
        for (int s = 0; s < 3; ++s)
          if (s != r) {
            con = A[s * 3 + r];
            A[s * 3 + r] = 0;
            for (int q = 0; q < 3; ++q) A[s * 3 + q] -= A[r * 3 + q] * con;
          }
      }
      const double bzx = h->hb[2][top] / h->hb[0][i], bzy = h->hb[2][top] / h->hb[1][j];
      const size_t m2 = (size_t)j * h->g.px + (i + XSH);
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) {
          double ab = 0, ac = 0;
          for (int q = 0; q < 3; ++q) {
            ab += A[r * 3 + q] * B[q * 3 + s];
            ac += A[r * 3 + q] * C[q * 3 + s];
          }
          out[(size_t)(r * 3 + s) * plane + m2] = (float)(-1 * ab * bzx);
          out[(size_t)(9 + r * 3 + s) * plane + m2] = (float)(-1 * ac * bzy);
        }
    }
}

// the receiver record of one step (after its four stages)
void launch_record(cgfd_solver *h) {
  ScaleSet s;
  for (int c = 0; c < NCOMP; ++c) s.sc[c] = std::ldexp(1.f, h->sexp[c]);
  if (h->elem == ELEM_F16)
    record_kernel<<<1, 256, 0, h->st>>>((const __half *)h->set[0], h->g.fstride, h->d_rcell,
                                        h->nrecv, h->d.nt, h->d_seis, h->d_step, s);
  else if (h->elem == ELEM_BF16)
    record_kernel<<<1, 256, 0, h->st>>>((const __nv_bfloat16 *)h->set[0], h->g.fstride,
                                        h->d_rcell, h->nrecv, h->d.nt, h->d_seis, h->d_step, s);
  else
    record_kernel<<<1, 256, 0, h->st>>>((const float *)h->set[0], h->g.fstride, h->d_rcell,
                                        h->nrecv, h->d.nt, h->d_seis, h->d_step, s);
}

// the per-component scales of the field sets (1 for FP32 storage)
ScaleSet field_scales(const cgfd_solver *h) {
  ScaleSet s;
  for (int c = 0; c < NCOMP; ++c) s.sc[c] = std::ldexp(1.f, h->sexp[c]);
  return s;
}

// the learned layer's correction of FW after a step
void launch_mlp(cgfd_solver *h, cudaStream_t st) {
  const size_t fs = h->g.fstride;
  launch_mlp_step(h->set[0], h->elem, fs, field_scales(h), h->media, h->media + 2 * fs,
                  h->d_mlp_cells, h->mlp_n, h->d_mlp_w, h->d_mlp_gain, h->mlp_width,
                  h->d_mlp_delta, st);
}

// the peak-velocity update of one step
void launch_pgv(cgfd_solver *h) {
  const float s0 = std::ldexp(1.f, h->sexp[0]), s1 = std::ldexp(1.f, h->sexp[1]),
              s2 = std::ldexp(1.f, h->sexp[2]);
  dim3 grid((h->d.ni + 127) / 128, h->d.nj);
  if (h->elem == ELEM_F16)
    pgv_kernel<<<grid, 128, 0, h->st>>>((const __half *)h->set[0], h->g, h->d_pgv, s0, s1, s2);
  else if (h->elem == ELEM_BF16)
    pgv_kernel<<<grid, 128, 0, h->st>>>((const __nv_bfloat16 *)h->set[0], h->g, h->d_pgv, s0,
                                        s1, s2);
  else
    pgv_kernel<<<grid, 128, 0, h->st>>>((const float *)h->set[0], h->g, h->d_pgv, s0, s1, s2);
}

StageArgs stage_args(cgfd_solver *h, int rk, int X, int Y, int Z, int in_set, int out_set) {
  StageArgs a{};
  a.g = h->g;
  a.rk = rk;
  a.X = X; a.Y = Y; a.Z = Z;
  a.h = (float)h->d.steph;
  a.adt = (rk < 3) ? (float)(RKA[rk] * h->d.stept) : 0.f;
  a.bdt = (float)(RKB[rk] * h->d.stept);
  a.tw_skip = h->d.kernel == CGFD_KERNEL_FUSED;
  a.rtw = (float)(RKB[0] / RKA[0]);
  a.in = h->set[in_set];
  a.fw = h->set[0];
  a.out = h->set[out_set];
  a.tw = h->set[3];
  a.elem = h->elem;
  for (int c = 0; c < NCOMP; ++c) {
    a.sc[c] = std::ldexp(1.f, h->sexp[c]);
    a.isc[c] = std::ldexp(1.f, -h->sexp[c]);
  }
  const size_t fs = h->g.fstride;
  a.lam2mu = h->media; a.mu = h->media + fs; a.irho = h->media + 2 * fs;
  a.zx = h->metric; a.zy = h->metric + fs; a.zz = h->metric + 2 * fs; a.jac = h->metric + 3 * fs;
  a.zzp = h->zzp;
  a.zu_end = h->zu_end;
  a.flat = h->flat;
  a.plain_interior = h->plain_interior;
  a.matv = h->matv;
  for (int q = 0; q < 3; ++q) {
    a.apd[q] = h->pmlp[q]; a.b[q] = h->pmlp[3 + q]; a.db[q] = h->pmlp[6 + q];
    if (h->aux[q]) {
      const size_t ss = (size_t)h->g.ncaux * h->g.astride[q];
      float *FA = h->aux[q], *A = h->aux[q] + ss, *TA = h->aux[q] + 2 * ss;
      a.ain[q] = (rk == 0) ? FA : A;
      a.afw[q] = FA;
      a.aout[q] = (rk == 3) ? FA : A;
      a.ta[q] = TA;
    }
  }
  return a;
}

// the stage kernels of the solver's kernel family
void dispatch_stage(cgfd_solver *h, const StageArgs &a, int in_set) {
  if (h->d.kernel == CGFD_KERNEL_SIMPLE)
    launch_stage_simple(a, h->st);
  else if (h->d.kernel == CGFD_KERNEL_FUSED)
    launch_stage_pair(h->plan, a, in_set, h->d_err, h->st, &h->side);
  else
    launch_stage_fused(h->plan, a, in_set, h->d_err, h->st);
}

// the sources of one stage (tindex < 0: from the device step counter)
SourceArgs source_args(const cgfd_solver *h, const StageArgs &a, int tindex) {
  SourceArgs s{};
  const int rk = a.rk;
  s.g = h->g;
  s.nmnt = h->nmnt; s.nfrc = h->nfrc;
  s.mcell = h->d_mcell; s.mcoef = h->d_mcoef; s.mstf = h->d_mstf; s.nstfm = h->nstfm;
  s.fcell = h->d_fcell; s.fcoef = h->d_fcoef; s.fstf = h->d_fstf; s.nstff = h->nstff;
  s.tinc = (rk == 0) ? 0 : (rk < 3 ? 1 : 2);
  s.tindex = tindex;
  s.step = h->d_step;
  s.adt = a.adt; s.bdt = a.bdt; s.tw_skip = a.tw_skip;
  s.out = a.out; s.tw = a.tw; s.rk = rk;
  s.elem = a.elem;
  for (int c = 0; c < NCOMP; ++c) s.isc[c] = a.isc[c];
  s.nfoc = h->nfoc; s.fnt = h->fnt;
  s.foccell = h->d_foccell; s.focmom = h->d_focmom;
  s.fdt = (float)h->fdt; s.dt = (float)h->d.stept; s.h = (float)h->d.steph;
  s.jac = h->metric + 3 * h->g.fstride;
  s.smooth = 0;
  for (int k = 0; k < 3; ++k)
    if (!h->smw[k].empty()) s.smooth |= 1u << k;
  s.nsp = h->sp_n;
  s.spcell = h->d_sp_cell; s.spoff = h->d_sp_off; s.sprow = h->d_sp_row;
  s.spcoef = h->d_sp_coef;
  return s;
}

// point sources, focal points, then the smoothed ones (separate launches:
// they may touch the same node)
int launch_stage_sources(cgfd_solver *h, const StageArgs &a, int tindex) {
  if (h->nmnt + h->nfrc + h->nfoc == 0) return CGFD_OK;
  const SourceArgs s = source_args(h, a, tindex);
  const int np = (h->smw[0].empty() ? h->nmnt : 0) + (h->smw[1].empty() ? h->nfrc : 0);
  if (np > 0) {
    launch_sources(s, h->st);
    CK(h, cudaGetLastError());
  }
  if (h->nfoc > 0 && h->smw[2].empty()) {
    launch_focal(s, h->st);
    CK(h, cudaGetLastError());
  }
  if (h->sp_n > 0) {
    launch_spread(s, h->st);
    CK(h, cudaGetLastError());
  }
  return CGFD_OK;
}

int launch_stage(cgfd_solver *h, int rk, int X, int Y, int Z, int in_set, int out_set,
                 int tindex) {
  StageArgs a = stage_args(h, rk, X, Y, Z, in_set, out_set);
  dispatch_stage(h, a, in_set);
  CK(h, cudaGetLastError());
  return launch_stage_sources(h, a, tindex);
}

// the four stages of one step of pattern p, reading tindex from the device
// step counter, then the receiver record
int enqueue_step(cgfd_solver *h, int p) {
  static const int ins[4] = {0, 1, 2, 1}, outs[4] = {1, 2, 1, 0};
  for (int rk = 0; rk < 4; ++rk) {
    const int *dd = DIRS[p][rk];
    int st = launch_stage(h, rk, dd[0], dd[1], dd[2], ins[rk], outs[rk], -1);
    if (st) return st;
  }
  if (h->mlp_n) {
    launch_mlp(h, h->st);
    CK(h, cudaGetLastError());
  }
  launch_record(h);
  CK(h, cudaGetLastError());
  if (h->d_pgv) {
    launch_pgv(h);
    CK(h, cudaGetLastError());
  }
  return CGFD_OK;
}

int build_graphs(cgfd_solver *h) {
  for (int p = 0; p < 4; ++p) {
    if (h->graph[p]) { cudaGraphExecDestroy(h->graph[p]); h->graph[p] = nullptr; }
    cudaGraph_t gr = nullptr;
    CK(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_step(h, p);
    cudaError_t e = cudaStreamEndCapture(h->st, &gr);
    if (st) { if (gr) cudaGraphDestroy(gr); return st; }
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&h->graph[p], gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
  }
  h->graphs_ok = true;
  return CGFD_OK;
}

}  // namespace

// --------------------------------- C ABI -----------------------------------
extern "C" {

int cgfd_create(const cgfd_desc *d, cgfd_solver **out) {
  CGFD_ABI_BEGIN
  if (!d || !out) return arg_fail(nullptr, "null argument");
  *out = nullptr;
  if (d->ni < 1 || d->nj < 1 || d->nk < 4 || !(d->steph > 0) || !(d->stept > 0) || d->nt < 0)
    return arg_fail(nullptr, "bad grid or step sizes");
  // far above any grid that fits one GPU; keeps every index product in range
  constexpr int MAX_AXIS = 1 << 20;
  if (d->ni > MAX_AXIS || d->nj > MAX_AXIS || d->nk > MAX_AXIS)
    return arg_fail(nullptr, "grid dimension above 2^20 cells");
  if (d->hybrid_grid != 1) return arg_fail(nullptr, "only hybrid_grid=1 (SimpleCar) is supported");
  for (int q = 0; q < 6; ++q)
    if (d->nabs[q] < 0) return arg_fail(nullptr, "negative nabs");
  if (d->nabs[5] != 0) return arg_fail(nullptr, "nabs[5] (top) must be 0: free surface");
  if (d->nabs[0] > d->ni || d->nabs[1] > d->ni - d->nabs[0] || d->nabs[2] > d->nj ||
      d->nabs[3] > d->nj - d->nabs[2] || d->nabs[4] > d->nk || d->nabs[5] > d->nk - d->nabs[4])
    return arg_fail(nullptr, "PML wider than the grid");
  if (d->con_index < LFD || d->con_index > d->nk + LFD - 1)
    return arg_fail(nullptr, "con_index must lie in [3, nk+2]");
  if (d->storage != CGFD_STORE_F32 && d->storage != CGFD_STORE_F16 &&
      d->storage != CGFD_STORE_BF16)
    return arg_fail(nullptr, "unknown storage type");
  if (d->storage != CGFD_STORE_F32 && d->kernel != CGFD_KERNEL_FUSED)
    return arg_fail(nullptr, "16-bit storage runs on the default kernel family only");
  if (d->kernel != CGFD_KERNEL_FUSED && d->kernel != CGFD_KERNEL_SIMPLE &&
      d->kernel != CGFD_KERNEL_SCALAR)
    return arg_fail(nullptr, "unknown kernel family");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    g_last_create_error = "no CUDA device";
    return CGFD_ERR_NODEVICE;
  }
  if (d->device < 0 || d->device >= ndev) return arg_fail(nullptr, "bad device ordinal");

  cgfd_solver *h = new cgfd_solver();
  h->d = *d;
  h->elem = d->storage == CGFD_STORE_F16    ? ELEM_F16
            : d->storage == CGFD_STORE_BF16 ? ELEM_BF16
                                            : ELEM_F32;
  Geom &g = h->g;
  g.ni = d->ni; g.nj = d->nj; g.nk = d->nk;
  g.px = (int)align_up((size_t)XO + d->ni + 4, 32);
  g.nyi = d->nj + 6; g.nzi = d->nk + 6;
  g.top = d->nk + LFD - 1;
  g.con = d->con_index;
  for (int q = 0; q < 6; ++q) g.nabs[q] = d->nabs[q];
  if (d->nabs[0] + d->nabs[1] > 0) {
    g.xaoff = d->nabs[0] + ((d->ni - d->nabs[1] - d->nabs[0]) % 4 + 4) % 4;
    g.nxa = (int)align_up((size_t)(g.xaoff + d->nabs[1]), 4);
  } else {
    g.xaoff = 0;
    g.nxa = 0;
  }
  g.nya = d->nabs[2] + d->nabs[3];
  g.nza = d->nabs[4] + d->nabs[5];
  g.plane = (size_t)g.px * g.nyi;
  g.fstride = align_up(g.plane * g.nzi, 64);
  g.astride[0] = align_up((size_t)g.nzi * g.nyi * g.nxa, 64);
  g.astride[1] = align_up((size_t)g.nzi * g.nya * g.px, 64);
  g.astride[2] = align_up((size_t)g.nza * g.nyi * g.px, 64);
  g.ncaux = (d->kernel == CGFD_KERNEL_FUSED) ? 6 : 9;
  if ((d->kernel == CGFD_KERNEL_SCALAR && !fused_supported(g)) ||
      (d->kernel == CGFD_KERNEL_FUSED && !pair_supported(g))) {
    delete h;
    return arg_fail(nullptr, "tiled kernel does not support this grid");
  }

  DevGuard guard(d->device);
  int st = CGFD_OK;
  auto alloc = [&](float **p, size_t n) -> int {
    cudaError_t e2 = cudaMalloc(p, n * sizeof(float));
    if (e2 != cudaSuccess) { cuda_fail(nullptr, e2, "cudaMalloc"); return CGFD_ERR_NOMEM; }
    e2 = cudaMemset(*p, 0, n * sizeof(float));
    if (e2 != cudaSuccess) { cuda_fail(nullptr, e2, "cudaMemset"); return CGFD_ERR_CUDA; }
    return CGFD_OK;
  };
  const size_t fs = g.fstride;
  // the four field sets, 9 components of fs elements of the storage type each
  if (!st) st = alloc((float **)&h->state, (4 * 9 * fs * elem_size(h->elem) + 3) / 4);
  if (!st) st = alloc(&h->media, 3 * fs);
  if (!st) st = alloc(&h->metric, 4 * fs);
  if (!st) st = alloc(&h->zzp, g.nzi);
  const size_t plen = align_up(g.px, 64) * 3 + align_up(g.nyi, 64) * 3 + align_up(g.nzi, 64) * 3;
  if (!st) st = alloc(&h->pml, plen);
  for (int q = 0; q < 3 && !st; ++q)
    if ((q == 0 ? g.nxa : q == 1 ? g.nya : g.nza) > 0)
      st = alloc(&h->aux[q], 3 * (size_t)g.ncaux * g.astride[q]);
  if (!st) st = alloc(&h->matv, 18 * g.plane);
  if (!st) {
    e = cudaMalloc(&h->d_step, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->d_step, 0, sizeof(int));
    h->nf_blocks = (int)nonfinite_blocks(9 * g.fstride);
    if (e == cudaSuccess)
      e = cudaMalloc(&h->d_partials, (h->nf_blocks + 1) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&h->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    cudaStream_t s2 = nullptr;
    cudaEvent_t e1 = nullptr, e2 = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
    h->side.stream = s2;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e1, cudaEventDisableTiming);
    h->side.fork = e1;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e2, cudaEventDisableTiming);
    h->side.join = e2;
    cudaStream_t s3 = nullptr;
    cudaEvent_t e3 = nullptr, e4 = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s3, cudaStreamNonBlocking);
    h->side.stream2 = s3;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e3, cudaEventDisableTiming);
    h->side.fork2 = e3;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&e4, cudaEventDisableTiming);
    h->side.join2 = e4;
    if (e != cudaSuccess) st = cuda_fail(nullptr, e, "setup");
  }
  if (st) {
    free_all(h);
    delete h;
    return st;
  }
  for (int q = 0; q < 4; ++q)
    h->set[q] = (char *)h->state + (size_t)q * 9 * fs * elem_size(h->elem);
  if (d->kernel == CGFD_KERNEL_FUSED || d->kernel == CGFD_KERNEL_SCALAR) {
    float *fsets[4] = {(float *)h->set[0], (float *)h->set[1], (float *)h->set[2],
                       (float *)h->set[3]};
    h->plan = (d->kernel == CGFD_KERNEL_FUSED)
                  ? pair_create_plan(g, h->elem, h->set, h->media, h->metric, h->aux)
                  : fused_create_plan(g, fsets, h->media, h->metric);
    if (!h->plan) {
      free_all(h);
      delete h;
      g_last_create_error = "cuTensorMapEncodeTiled failed";
      return CGFD_ERR_CUDA;
    }
  }
  {
    float *p = h->pml;
    const size_t lx = align_up(g.px, 64), ly = align_up(g.nyi, 64), lz = align_up(g.nzi, 64);
    for (int t = 0; t < 3; ++t) {
      h->pmlp[3 * t + 0] = p; p += lx;
      h->pmlp[3 * t + 1] = p; p += ly;
      h->pmlp[3 * t + 2] = p; p += lz;
    }
  }
  h->wcur = 0;
  *out = h;
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

int cgfd_destroy(cgfd_solver *h) {
  CGFD_ABI_BEGIN
  if (!h) return CGFD_OK;
  {
    DevGuard guard(h->d.device);
    if (h->st) cudaStreamSynchronize(h->st);
    free_all(h);
  }
  delete h;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_last_error(const cgfd_solver *h, char *buf, size_t len) {
  CGFD_ABI_BEGIN
  if (!buf || !len) return CGFD_ERR_ARG;
  std::snprintf(buf, len, "%s", h ? h->err.c_str() : g_last_create_error.c_str());
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_upload_metric(cgfd_solver *h, const double *zx, const double *zy, const double *zz,
                       const double *jac) {
  CGFD_ABI_BEGIN
  if (!h || !zx || !zy || !zz || !jac) return arg_fail(h, "null argument");
  DevGuard guard(h->d.device);
  const long n = ref_n(h);
  const int nx = h->d.ni + 6, ny = h->d.nj + 6, nz = h->d.nk + 6;
  (void)n;
  const double *src[4] = {zx, zy, zz, jac};
  float *dst[4];
  for (int q = 0; q < 4; ++q) dst[q] = h->metric + (size_t)q * h->g.fstride;
  // Checked on the converted (stored) values of the valid cells, inside the
  // conversion pass that streams every value anyway:
  //  * trivial metric (zeta = (0,0,1), J = 1) everywhere: the flat path.
  //    Metric values in ghost cells only ever multiply zero wavefield values
  //    or are replaced by the traction image, so they do not matter;
  //  * per plane below ConIndex, whether zeta_z is one value on every valid
  //    cell (that of column (3, 3)): the tiled kernels take it from a
  //    per-plane table instead of loading the plane's metric tile (zeta_x
  //    and zeta_y are not used below ConIndex).
  const int kmax = std::min(h->d.nk + LFD, h->g.con);
  std::vector<float> zref(nz, 0.f);
  for (int k = LFD; k < kmax; ++k) zref[k] = (float)zz[((long)LFD * ny + LFD) * nz + k];
  std::atomic<bool> flat{true};
  std::unique_ptr<std::atomic<unsigned char>[]> differs(new std::atomic<unsigned char>[nz]);
  for (int k = 0; k < nz; ++k) differs[k].store(0, std::memory_order_relaxed);
  const float triv[4] = {0.f, 0.f, 1.f, 1.f};
  int st = upload_fields(
      h, 4,
      [&](int a, long b, long e, float *o) {
        const double *s = src[a];
        for (long t = b; t < e; ++t) o[t - b] = (float)s[t];
        bool nonflat = false;
        std::vector<unsigned char> dk(a == 2 ? nz : 0, 0);
        // runs of one z-column within [b, e)
        for (long t = b; t < e;) {
          const long col = t / nz;
          const int k0 = (int)(t - col * nz);
          const long t1 = std::min(e, (col + 1) * nz);
          const int i = (int)(col / ny), j = (int)(col % ny);
          if (i >= LFD && i < h->d.ni + LFD && j >= LFD && j < h->d.nj + LFD) {
            const float *c = o + (t - b) - k0;  // c[k]: the column's value at k
            const int kb = std::max(k0, LFD), ke = std::min(k0 + (int)(t1 - t), h->d.nk + LFD);
            for (int k = kb; k < ke; ++k) nonflat |= c[k] != triv[a];
            if (a == 2)
              for (int k = kb; k < std::min(ke, kmax); ++k) dk[k] |= c[k] != zref[k];
          }
          t = t1;
        }
        if (nonflat) flat.store(false, std::memory_order_relaxed);
        for (int k = 0; k < (int)dk.size(); ++k)
          if (dk[k]) differs[k].store(1, std::memory_order_relaxed);
      },
      dst);
  if (st) return st;
  h->flat = flat;
  std::vector<float> zzp(h->g.nzi, 0.f);
  std::vector<char> same(h->g.nzi, 0);
  for (int k = LFD; k < kmax; ++k) {
    same[k] = !differs[k].load(std::memory_order_relaxed);
    if (same[k]) zzp[k] = zref[k];
  }
  int zu_end = LFD;
  while (zu_end < kmax && same[zu_end]) ++zu_end;
  CK(h, cudaMemcpy(h->zzp, zzp.data(), zzp.size() * sizeof(float), cudaMemcpyHostToDevice));
  h->zu_end = zu_end;
  h->top_zeta.assign(3 * (size_t)nx * ny, 0.0);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const long t = ((long)i * ny + j) * nz + h->g.top;
      const size_t t2 = (size_t)i * ny + j;
      h->top_zeta[t2] = zx[t];
      h->top_zeta[(size_t)nx * ny + t2] = zy[t];
      h->top_zeta[2 * (size_t)nx * ny + t2] = zz[t];
    }
  h->have_metric = true;
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_upload_media(cgfd_solver *h, const float *alpha, const float *beta, const float *rho) {
  CGFD_ABI_BEGIN
  if (!h || !alpha || !beta || !rho) return arg_fail(h, "null argument");
  DevGuard guard(h->d.device);
  const long n = ref_n(h);
  const int nx = h->d.ni + 6, ny = h->d.nj + 6, nz = h->d.nk + 6;
  (void)n;
  // (lambda + 2 mu, mu, 1/rho) as FP32 from double products; the valid
  // cells must have a positive density, checked in the 1/rho pass (a failed
  // check leaves the solver without media)
  float *dst[3] = {h->media, h->media + h->g.fstride, h->media + 2 * h->g.fstride};
  std::atomic<bool> bad{false};
  int st = upload_fields(
      h, 3,
      [&](int a, long b, long e, float *o) {
        for (long t = b; t < e; ++t) {
          const double r = rho[t];
          o[t - b] = a == 0   ? (float)(r * (double)alpha[t] * alpha[t])
                     : a == 1 ? (float)(r * (double)beta[t] * beta[t])
                              : (r != 0.0 ? (float)(1.0 / r) : 0.f);
        }
        if (a != 2) return;
        bool nonpos = false;
        for (long t = b; t < e;) {  // runs of one z-column within [b, e)
          const long col = t / nz;
          const int k0 = (int)(t - col * nz);
          const long t1 = std::min(e, (col + 1) * nz);
          const int i = (int)(col / ny), j = (int)(col % ny);
          if (i >= LFD && i < h->d.ni + LFD && j >= LFD && j < h->d.nj + LFD) {
            const float *r = rho + t - k0;
            const int ke = std::min(k0 + (int)(t1 - t), h->d.nk + LFD);
            for (int k = std::max(k0, LFD); k < ke; ++k) nonpos |= !(r[k] > 0.f);
          }
          t = t1;
        }
        if (nonpos) bad.store(true, std::memory_order_relaxed);
      },
      dst);
  if (st) return st;
  if (bad) {
    h->have_media = false;
    invalidate(h);
    return arg_fail(h, "non-positive density");
  }
  h->top_alpha.assign((size_t)nx * ny, 0.0);
  h->top_beta.assign((size_t)nx * ny, 0.0);
  h->top_rho.assign((size_t)nx * ny, 0.0);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      const long t = ((long)i * ny + j) * nz + h->g.top;
      h->top_alpha[(size_t)i * ny + j] = alpha[t];
      h->top_beta[(size_t)i * ny + j] = beta[t];
      h->top_rho[(size_t)i * ny + j] = rho[t];
    }
  h->have_media = true;
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_upload_pml(cgfd_solver *h, const double *apdx, const double *apdy, const double *apdz,
                    const double *bx, const double *by, const double *bz, const double *dbx,
                    const double *dby, const double *dbz) {
  CGFD_ABI_BEGIN
  if (!h || !apdx || !apdy || !apdz || !bx || !by || !bz || !dbx || !dby || !dbz)
    return arg_fail(h, "null argument");
  DevGuard guard(h->d.device);
  const int n3[3] = {h->d.ni + 6, h->d.nj + 6, h->d.nk + 6};
  const int len[3] = {h->g.px, h->g.nyi, h->g.nzi};
  const int off[3] = {XSH, 0, 0};  // internal index = reference index + off
  const double *src[9] = {apdx, apdy, apdz, bx, by, bz, dbx, dby, dbz};
  for (int q = 0; q < 9; ++q) {
    const int ax = q % 3;
    // B defaults to 1 (no stretching) outside the reference range
    std::vector<float> v(len[ax], q / 3 == 1 ? 1.f : 0.f);
    for (int t = 0; t < n3[ax]; ++t) {
      if (q / 3 == 1 && !(src[q][t] > 0.0)) return arg_fail(h, "PML B must be positive");
      v[t + off[ax]] = (float)src[q][t];
    }
    CK(h, cudaMemcpy(h->pmlp[q], v.data(), len[ax] * sizeof(float), cudaMemcpyHostToDevice));
  }
  for (int ax = 0; ax < 3; ++ax) h->hb[ax].assign(src[3 + ax], src[3 + ax] + n3[ax]);
  // outside the layers the factors must be B = 1, DB = APD = 0 for the
  // kernels' interior path; otherwise every cell takes the general path
  bool plain = true;
  const int nv[3] = {h->d.ni, h->d.nj, h->d.nk};
  for (int ax = 0; ax < 3; ++ax)
    for (int t = 3 + h->d.nabs[2 * ax]; t < 3 + nv[ax] - h->d.nabs[2 * ax + 1]; ++t)
      if (src[3 + ax][t] != 1.0 || src[6 + ax][t] != 0.0 || src[ax][t] != 0.0) plain = false;
  h->plain_interior = plain;
  h->have_pml = true;
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

static int upload_points(cgfd_solver *h, int n, const int *loc, int ncoef, const float *coef,
                         int nstf, const float *stf, std::vector<int> &hloc,
                         std::vector<float> &hcoef, std::vector<float> &hstf, int *&dcell,
                         float *&dstf, int &cnt, int &cnstf) {
  if (n < 0 || (n > 0 && (!loc || !coef || !stf || nstf < 1))) return arg_fail(h, "bad sources");
  for (int q = 0; q < n; ++q)
    if (!valid_loc(h, loc + 3 * q)) return arg_fail(h, "source outside the valid grid");
  DevGuard guard(h->d.device);
  if (dcell) { cudaFree(dcell); dcell = nullptr; }
  if (dstf) { cudaFree(dstf); dstf = nullptr; }
  hloc.assign(loc, loc + 3 * n);
  hcoef.assign(coef, coef + (size_t)ncoef * n);
  if (n > 0) hstf.assign(stf, stf + (size_t)n * nstf);
  else hstf.clear();
  cnt = n;
  cnstf = nstf;
  if (n > 0) {
    std::vector<int> cells(n);
    for (int q = 0; q < n; ++q) cells[q] = cell_of(h, loc + 3 * q);
    CK(h, cudaMalloc(&dcell, n * sizeof(int)));
    CK(h, cudaMemcpy(dcell, cells.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CK(h, cudaMalloc(&dstf, (size_t)n * nstf * sizeof(float)));
    CK(h, cudaMemcpy(dstf, stf, (size_t)n * nstf * sizeof(float), cudaMemcpyHostToDevice));
  }
  invalidate(h);
  return CGFD_OK;
}

int cgfd_upload_moments(cgfd_solver *h, int n, const int *loc, const float *m6, int nstf,
                        const float *stf) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  h->smw[0].clear();
  return upload_points(h, n, loc, 6, m6, nstf, stf, h->mloc, h->m6, h->hmstf, h->d_mcell,
                       h->d_mstf, h->nmnt, h->nstfm);
  CGFD_ABI_END(h)
}

int cgfd_upload_forces(cgfd_solver *h, int n, const int *loc, const float *f3, int nstf,
                       const float *stf) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  h->smw[1].clear();
  return upload_points(h, n, loc, 3, f3, nstf, stf, h->floc, h->f3, h->hfstf, h->d_fcell,
                       h->d_fstf, h->nfrc, h->nstff);
  CGFD_ABI_END(h)
}

int cgfd_upload_focal(cgfd_solver *h, int n, const int *loc, int fnt, double fdt,
                      const float *mom) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (n < 0 || (n > 0 && (!loc || !mom || fnt < 1 || !(fdt > 0.0))))
    return arg_fail(h, "bad focal sources");
  for (int q = 0; q < n; ++q)
    if (!valid_loc(h, loc + 3 * q)) return arg_fail(h, "focal source outside the valid grid");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  h->smw[2].clear();
  if (h->d_foccell) { cudaFree(h->d_foccell); h->d_foccell = nullptr; }
  if (h->d_focmom) { cudaFree(h->d_focmom); h->d_focmom = nullptr; }
  h->nfoc = 0;
  h->focloc.clear();
  h->hfocmom.clear();
  if (n > 0) {
    const size_t nm = (size_t)6 * n * fnt;
    std::vector<int> cells(n);
    for (int q = 0; q < n; ++q) cells[q] = cell_of(h, loc + 3 * q);
    CK(h, cudaMalloc(&h->d_foccell, n * sizeof(int)));
    CK(h, cudaMemcpy(h->d_foccell, cells.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CK(h, cudaMalloc(&h->d_focmom, nm * sizeof(float)));
    CK(h, cudaMemcpy(h->d_focmom, mom, nm * sizeof(float), cudaMemcpyHostToDevice));
    h->focloc.assign(loc, loc + 3 * n);
    h->hfocmom.assign(mom, mom + nm);
    h->nfoc = n;
    h->fnt = fnt;
    h->fdt = fdt;
  }
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_set_source_smoothing(cgfd_solver *h, int kind, int n, const double *weights) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (kind < 0 || kind > 2) return arg_fail(h, "source smoothing: kind must be 0, 1 or 2");
  const int have = kind == 0 ? h->nmnt : (kind == 1 ? h->nfrc : h->nfoc);
  if (!weights || n == 0) {
    if (n != 0) return arg_fail(h, "source smoothing: weights missing");
    h->smw[kind].clear();
  } else {
    if (n != have) return arg_fail(h, "source smoothing: n differs from the uploaded sources");
    // the spread list packs (kind, source) into one int: kind << 28 | q
    if (n >= (1 << 28)) return arg_fail(h, "source smoothing: too many sources");
    for (size_t t = 0; t < (size_t)343 * n; ++t)
      if (!std::isfinite(weights[t])) return arg_fail(h, "source smoothing: weights not finite");
    h->smw[kind].assign(weights, weights + (size_t)343 * n);
  }
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_set_receivers(cgfd_solver *h, int n, const int *loc) {
  CGFD_ABI_BEGIN
  if (!h || n < 0 || (n > 0 && !loc)) return arg_fail(h, "bad receivers");
  for (int q = 0; q < n; ++q)
    if (!valid_loc(h, loc + 3 * q)) return arg_fail(h, "receiver outside the valid grid");
  DevGuard guard(h->d.device);
  if (h->d_rcell) { cudaFree(h->d_rcell); h->d_rcell = nullptr; }
  if (h->d_seis) { cudaFree(h->d_seis); h->d_seis = nullptr; }
  h->nrecv = n;
  if (n > 0) {
    std::vector<int> cells(n);
    for (int q = 0; q < n; ++q) cells[q] = cell_of(h, loc + 3 * q);
    CK(h, cudaMalloc(&h->d_rcell, n * sizeof(int)));
    CK(h, cudaMemcpy(h->d_rcell, cells.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    const size_t ns = (size_t)9 * n * (h->d.nt > 0 ? h->d.nt : 1);
    CK(h, cudaMalloc(&h->d_seis, ns * sizeof(float)));
    CK(h, cudaMemset(h->d_seis, 0, ns * sizeof(float)));
  }
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

// sets the per-component scale exponents of 16-bit storage, rescaling the
// stored fields so that the values they stand for do not change
static int apply_scales(cgfd_solver *h, const int *e) {
  for (int c = 0; c < NCOMP; ++c) {
    if (e[c] == h->sexp[c]) continue;
    const float f = std::ldexp(1.f, h->sexp[c] - e[c]);
    if (h->elem == ELEM_F16)
      rescale_kernel<<<592, 256, 0, h->st>>>((__half *)h->state, h->g.fstride, c, f);
    else if (h->elem == ELEM_BF16)
      rescale_kernel<<<592, 256, 0, h->st>>>((__nv_bfloat16 *)h->state, h->g.fstride, c, f);
    CK(h, cudaGetLastError());
    h->sexp[c] = e[c];
  }
  CK(h, cudaStreamSynchronize(h->st));
  return CGFD_OK;
}

int cgfd_set_field_scales(cgfd_solver *h, const int *exp2) {
  CGFD_ABI_BEGIN
  if (!h || !exp2) return arg_fail(h, "null argument");
  for (int c = 0; c < NCOMP; ++c)
    if (exp2[c] < -60 || exp2[c] > 60) return arg_fail(h, "scale exponent out of range");
  if (h->elem == ELEM_F32) {
    for (int c = 0; c < NCOMP; ++c)
      if (exp2[c] != 0) return arg_fail(h, "scales apply to 16-bit storage only");
    return CGFD_OK;
  }
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  int st = apply_scales(h, exp2);
  if (st) return st;
  h->user_scales = true;
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_get_field_scales(cgfd_solver *h, int *exp2) {
  CGFD_ABI_BEGIN
  if (!h || !exp2) return arg_fail(h, "null argument");
  for (int c = 0; c < NCOMP; ++c) exp2[c] = h->sexp[c];
  return CGFD_OK;
  CGFD_ABI_END(h)
}

}  // extern "C"

namespace {

// The spread list of the smoothed sources: every (source, valid node of its
// 7^3 block) pair with its coefficients, ordered by node (stable, so the
// entries of a node stay in kind, source, block order), and the offsets of
// each node's entries.  J and 1/rho come from one download of each.
int build_spread(cgfd_solver *h) {
  for (auto p : {(void **)&h->d_sp_cell, (void **)&h->d_sp_off, (void **)&h->d_sp_row,
                 (void **)&h->d_sp_coef})
    if (*p) { cudaFree(*p); *p = nullptr; }
  h->sp_n = 0;
  if (h->smw[0].empty() && h->smw[1].empty() && h->smw[2].empty()) return CGFD_OK;
  const size_t fs = h->g.fstride;
  std::vector<float> jac(fs), irho(fs);
  CK(h, cudaMemcpy(jac.data(), h->metric + 3 * fs, fs * sizeof(float), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(irho.data(), h->media + 2 * fs, fs * sizeof(float), cudaMemcpyDeviceToHost));
  const double h3 = h->d.steph * h->d.steph * h->d.steph;
  struct Ent {
    int cell, row;
    float c[6];
  };
  std::vector<Ent> ents;
  const int nk[3] = {h->nmnt, h->nfrc, h->nfoc};
  const std::vector<int> *locs[3] = {&h->mloc, &h->floc, &h->focloc};
  for (int kind = 0; kind < 3; ++kind) {
    if (h->smw[kind].empty()) continue;
    for (int q = 0; q < nk[kind]; ++q) {
      const int *l = &(*locs[kind])[3 * q];
      for (int a = 0; a < 7; ++a)
        for (int b = 0; b < 7; ++b)
          for (int c = 0; c < 7; ++c) {
            const int ijk[3] = {l[0] + a - 3, l[1] + b - 3, l[2] + c - 3};
            if (!valid_loc(h, ijk)) continue;
            const double w = h->smw[kind][(size_t)343 * q + (a * 7 + b) * 7 + c];
            Ent e{};
            e.cell = cell_of(h, ijk);
            e.row = (kind << 28) | q;
            const double A = w / (h3 * (double)jac[e.cell]);
            if (kind == 0) {
              for (int m = 0; m < 6; ++m) e.c[m] = (float)(h->m6[6 * q + m] * A);
            } else if (kind == 1) {
              double F = A * (double)irho[e.cell];
              if (ijk[2] == h->g.top) F *= 2.0;
              for (int m = 0; m < 3; ++m) e.c[m] = (float)(h->f3[3 * q + m] * F);
            } else {
              e.c[0] = (float)A;
            }
            ents.push_back(e);
          }
    }
  }
  std::stable_sort(ents.begin(), ents.end(),
                   [](const Ent &x, const Ent &y) { return x.cell < y.cell; });
  std::vector<int> cells, off, rows(ents.size());
  std::vector<float> coef((size_t)6 * ents.size());
  for (size_t e = 0; e < ents.size(); ++e) {
    if (e == 0 || ents[e].cell != ents[e - 1].cell) {
      cells.push_back(ents[e].cell);
      off.push_back((int)e);
    }
    rows[e] = ents[e].row;
    for (int m = 0; m < 6; ++m) coef[6 * e + m] = ents[e].c[m];
  }
  off.push_back((int)ents.size());
  if (cells.empty()) return CGFD_OK;
  CK(h, cudaMalloc(&h->d_sp_cell, cells.size() * sizeof(int)));
  CK(h, cudaMalloc(&h->d_sp_off, off.size() * sizeof(int)));
  CK(h, cudaMalloc(&h->d_sp_row, rows.size() * sizeof(int)));
  CK(h, cudaMalloc(&h->d_sp_coef, coef.size() * sizeof(float)));
  CK(h, cudaMemcpy(h->d_sp_cell, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(h->d_sp_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(h->d_sp_row, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(h->d_sp_coef, coef.data(), coef.size() * sizeof(float), cudaMemcpyHostToDevice));
  h->sp_n = (int)cells.size();
  return CGFD_OK;
}

}  // namespace

extern "C" {

int cgfd_prepare(cgfd_solver *h) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (!(h->have_metric && h->have_media && h->have_pml)) {
    h->err = "metric, media and PML must be uploaded before stepping";
    return CGFD_ERR_STATE;
  }
  if (h->prepared && h->graphs_ok) return CGFD_OK;
  DevGuard guard(h->d.device);
  std::vector<float> mv;
  surface_matrices(h, mv);
  CK(h, cudaMemcpy(h->matv, mv.data(), mv.size() * sizeof(float), cudaMemcpyHostToDevice));
  // source coefficients from the device copies of jac and 1/rho
  const double h3 = h->d.steph * h->d.steph * h->d.steph;
  auto cell_value = [&](const float *base, int cell, float *v) {
    return cudaMemcpy(v, base + cell, sizeof(float), cudaMemcpyDeviceToHost);
  };
  const size_t fs = h->g.fstride;
  if (h->d_mcoef) { cudaFree(h->d_mcoef); h->d_mcoef = nullptr; }
  if (h->d_fcoef) { cudaFree(h->d_fcoef); h->d_fcoef = nullptr; }
  if (h->nmnt) {
    std::vector<float> c(6 * h->nmnt);
    for (int q = 0; q < h->nmnt; ++q) {
      float jac = 1.f;
      CK(h, cell_value(h->metric + 3 * fs, cell_of(h, &h->mloc[3 * q]), &jac));
      const double A = 1.0 / (h3 * jac);
      for (int m = 0; m < 6; ++m) c[6 * q + m] = (float)(h->m6[6 * q + m] * A);
    }
    CK(h, cudaMalloc(&h->d_mcoef, c.size() * sizeof(float)));
    CK(h, cudaMemcpy(h->d_mcoef, c.data(), c.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (h->nfrc) {
    std::vector<float> c(3 * h->nfrc);
    for (int q = 0; q < h->nfrc; ++q) {
      const int cell = cell_of(h, &h->floc[3 * q]);
      float jac = 1.f, irho = 1.f;
      CK(h, cell_value(h->metric + 3 * fs, cell, &jac));
      CK(h, cell_value(h->media + 2 * fs, cell, &irho));
      double A = irho / (h3 * jac);
      if (h->floc[3 * q + 2] == h->g.top) A *= 2.0;
      for (int m = 0; m < 3; ++m) c[3 * q + m] = (float)(h->f3[3 * q + m] * A);
    }
    CK(h, cudaMalloc(&h->d_fcoef, c.size() * sizeof(float)));
    CK(h, cudaMemcpy(h->d_fcoef, c.data(), c.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  int sst = build_spread(h);
  if (sst) return sst;
  if (h->elem == ELEM_F16 && !h->user_scales) {
    // FP16 scale exponents from an estimate of the peak magnitudes: the
    // stress a moment source builds at its cell is bounded by its rate
    // coefficient M/(h^3 J) times the integral of |STF|; velocities follow
    // through the impedance rho*vs (sigma ~ rho vs v), and a force's velocity
    // rate f/(h^3 J rho) the other way round (sigma ~ rho vp v).  The peak is
    // put at 2^12 stored units, 2^4 below the FP16 maximum.
    const double dt2 = 0.5 * h->d.stept;
    double sT = 0, sV = 0;
    auto stf_int = [&](const std::vector<float> &stf, int q, int n) {
      double a = 0;
      for (int t = 0; t < n; ++t) a += std::fabs(stf[(size_t)q * n + t]) * dt2;
      return a;
    };
    for (int q = 0; q < h->nmnt; ++q) {
      const int cell = cell_of(h, &h->mloc[3 * q]);
      float jac = 1.f, mu = 0.f, irho = 1.f;
      CK(h, cell_value(h->metric + 3 * fs, cell, &jac));
      CK(h, cell_value(h->media + fs, cell, &mu));
      CK(h, cell_value(h->media + 2 * fs, cell, &irho));
      double m = 0;
      for (int c = 0; c < 6; ++c) m = std::fmax(m, std::fabs(h->m6[6 * q + c]));
      const double sig = m / (h3 * jac) * stf_int(h->hmstf, q, h->nstfm);
      const double z = std::sqrt(std::fmax((double)mu, 1e-30) / irho);  // rho vs
      sT = std::fmax(sT, sig);
      sV = std::fmax(sV, sig / z);
    }
    for (int q = 0; q < h->nfrc; ++q) {
      const int cell = cell_of(h, &h->floc[3 * q]);
      float jac = 1.f, l2m = 0.f, irho = 1.f;
      CK(h, cell_value(h->metric + 3 * fs, cell, &jac));
      CK(h, cell_value(h->media, cell, &l2m));
      CK(h, cell_value(h->media + 2 * fs, cell, &irho));
      double f = 0;
      for (int c = 0; c < 3; ++c) f = std::fmax(f, std::fabs(h->f3[3 * q + c]));
      const double v = 2.0 * f * irho / (h3 * jac) * stf_int(h->hfstf, q, h->nstff);
      sV = std::fmax(sV, v);
      sT = std::fmax(sT, v * std::sqrt(std::fmax((double)l2m, 1e-30) / irho));  // rho vp
    }
    if (h->nfoc > 0) {
      // focal points: the series are moment rates added to the stress RHS;
      // the point with the largest integral of its largest component bounds
      // the stress it builds (points are assumed not to pile up in a cell)
      int qmax = 0;
      double imax = 0;
      for (int q = 0; q < h->nfoc; ++q) {
        double im = 0;
        for (int m = 0; m < 6; ++m) {
          double a = 0;
          const float *ser = &h->hfocmom[((size_t)m * h->nfoc + q) * h->fnt];
          for (int t = 0; t < h->fnt; ++t) a += std::fabs(ser[t]) * h->fdt;
          im = std::fmax(im, a);
        }
        if (im > imax) { imax = im; qmax = q; }
      }
      const int cell = cell_of(h, &h->focloc[3 * qmax]);
      float jac = 1.f, mu = 0.f, irho = 1.f;
      CK(h, cell_value(h->metric + 3 * fs, cell, &jac));
      CK(h, cell_value(h->media + fs, cell, &mu));
      CK(h, cell_value(h->media + 2 * fs, cell, &irho));
      const double sig = imax / (h3 * jac);
      sT = std::fmax(sT, sig);
      sV = std::fmax(sV, sig / std::sqrt(std::fmax((double)mu, 1e-30) / irho));
    }
    auto ex = [](double peak) {
      return peak > 0 ? (int)std::ceil(std::log2(peak / 4096.0)) : 0;
    };
    int e[NCOMP];
    for (int c = 0; c < NCOMP; ++c) e[c] = c < 3 ? ex(sV) : ex(sT);
    for (int c = 0; c < NCOMP; ++c) e[c] = e[c] < -60 ? -60 : (e[c] > 60 ? 60 : e[c]);
    int st2 = apply_scales(h, e);
    if (st2) return st2;
  }
  h->prepared = true;
  int st = build_graphs(h);
  if (st) return st;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_step(cgfd_solver *h, int n_steps) {
  CGFD_ABI_BEGIN
  if (!h || n_steps < 0) return arg_fail(h, "bad arguments");
  int st = cgfd_prepare(h);
  if (st) return st;
  const int last = h->steps + n_steps - 1;
  if (n_steps > 0) {
    if (h->nrecv && last >= h->d.nt) return arg_fail(h, "more steps than the seismogram buffer (nt)");
    if ((h->nmnt && 2 * last + 2 >= h->nstfm) || (h->nfrc && 2 * last + 2 >= h->nstff))
      return arg_fail(h, "source time function too short for the requested steps");
  }
  DevGuard guard(h->d.device);
  CK(h, cudaMemcpyAsync(h->d_step, &h->steps, sizeof(int), cudaMemcpyHostToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  for (int s = 0; s < n_steps; ++s) {
    CK(h, cudaGraphLaunch(h->graph[h->steps % 4], h->st));
    h->steps++;
  }
  h->wcur = 0;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_step_timed(cgfd_solver *h, int n_steps, float *ms, float *stage_ms) {
  CGFD_ABI_BEGIN
  if (!h || n_steps < 1 || !ms) return arg_fail(h, "bad arguments");
  int st = cgfd_prepare(h);
  if (st) return st;
  const int last = h->steps + n_steps - 1;
  if (h->nrecv && last >= h->d.nt) return arg_fail(h, "more steps than the seismogram buffer (nt)");
  if ((h->nmnt && 2 * last + 2 >= h->nstfm) || (h->nfrc && 2 * last + 2 >= h->nstff))
    return arg_fail(h, "source time function too short for the requested steps");
  DevGuard guard(h->d.device);
  CK(h, cudaMemcpyAsync(h->d_step, &h->steps, sizeof(int), cudaMemcpyHostToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  cudaEvent_t e0, e1;
  CK(h, cudaEventCreate(&e0));
  CK(h, cudaEventCreate(&e1));
  std::vector<cudaEvent_t> ev;
  if (stage_ms) {
    ev.resize(8 * (size_t)n_steps);
    for (auto &e : ev) CK(h, cudaEventCreate(&e));
  }
  CK(h, cudaEventRecord(e0, h->st));
  static const int ins[4] = {0, 1, 2, 1}, outs[4] = {1, 2, 1, 0};
  for (int s = 0; s < n_steps; ++s) {
    const int p = h->steps % 4;
    if (!stage_ms) {
      CK(h, cudaGraphLaunch(h->graph[p], h->st));
    } else {
      for (int rk = 0; rk < 4; ++rk) {
        const int *dd = DIRS[p][rk];
        StageArgs a = stage_args(h, rk, dd[0], dd[1], dd[2], ins[rk], outs[rk]);
        CK(h, cudaEventRecord(ev[8 * (size_t)s + 2 * rk], h->st));
        dispatch_stage(h, a, ins[rk]);
        CK(h, cudaGetLastError());
        CK(h, cudaEventRecord(ev[8 * (size_t)s + 2 * rk + 1], h->st));
        // sources exactly as in the graph
        int sst = launch_stage_sources(h, a, -1);
        if (sst) return sst;
      }
      if (h->mlp_n) {
        launch_mlp(h, h->st);
        CK(h, cudaGetLastError());
      }
      launch_record(h);
      CK(h, cudaGetLastError());
      if (h->d_pgv) {
        launch_pgv(h);
        CK(h, cudaGetLastError());
      }
    }
    h->steps++;
  }
  CK(h, cudaEventRecord(e1, h->st));
  CK(h, cudaEventSynchronize(e1));
  CK(h, cudaEventElapsedTime(ms, e0, e1));
  if (stage_ms) {
    double sum = 0;
    for (size_t q = 0; q < ev.size(); q += 2) {
      float t = 0;
      CK(h, cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
      sum += t;
    }
    *stage_ms = (float)(sum / (ev.size() / 2));
    for (auto &e : ev) cudaEventDestroy(e);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->wcur = 0;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_rk_stage(cgfd_solver *h, int rk, int curr_t, int X, int Y, int Z) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (rk < 0 || rk > 3 || (X != 1 && X != -1) || (Y != 1 && Y != -1) || (Z != 1 && Z != -1) ||
      curr_t < 0)
    return arg_fail(h, "bad stage arguments");
  int st = cgfd_prepare(h);
  if (st) return st;
  const int tinc = (rk == 0) ? 0 : (rk < 3 ? 1 : 2);
  const int tindex = 2 * curr_t + tinc;
  if ((h->nmnt && tindex >= h->nstfm) || (h->nfrc && tindex >= h->nstff))
    return arg_fail(h, "source time function too short for this step");
  DevGuard guard(h->d.device);
  // input: FW for rk 0, else the last stage output; output: the other W set
  const int in = (rk == 0) ? 0 : h->wcur;
  int out;
  if (rk == 3) out = 0;
  else out = (in == 1) ? 2 : 1;
  if (rk == 3 && in == 0) return arg_fail(h, "stage 3 needs a previous stage output");
  st = launch_stage(h, rk, X, Y, Z, in, out, tindex);
  if (st) return st;
  if (rk == 0 && h->d.kernel == CGFD_KERNEL_FUSED) {  // tW elision: materialise tW
    const float r = (float)(RKB[0] / RKA[0]);
    if (h->elem == ELEM_F16)
      rebuild_tw_kernel<<<592, 256, 0, h->st>>>(h->g, (const __half *)h->set[0],
                                                (const __half *)h->set[out], (__half *)h->set[3], r);
    else if (h->elem == ELEM_BF16)
      rebuild_tw_kernel<<<592, 256, 0, h->st>>>(h->g, (const __nv_bfloat16 *)h->set[0],
                                                (const __nv_bfloat16 *)h->set[out],
                                                (__nv_bfloat16 *)h->set[3], r);
    else
      rebuild_tw_kernel<<<592, 256, 0, h->st>>>(h->g, (const float *)h->set[0],
                                                (const float *)h->set[out], (float *)h->set[3], r);
    CK(h, cudaGetLastError());
  }
  h->wcur = out;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_sync(cgfd_solver *h, double timeout_s) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  DevGuard guard(h->d.device);
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(h->st);
    if (e == cudaSuccess) {
      int flag = 0;
      CK(h, cudaMemcpy(&flag, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
      if (flag) {
        h->err = flag == 2 ? "stage kernel alignment self-check failed (no copy issued)"
                           : "a bounded wait inside a stage kernel expired";
        return flag == 2 ? CGFD_ERR_CUDA : CGFD_ERR_TIMEOUT;
      }
      return CGFD_OK;
    }
    if (e != cudaErrorNotReady) return cuda_fail(h, e, "cudaStreamQuery");
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (timeout_s >= 0 && el > timeout_s) {
      h->err = "timeout waiting for the device";
      return CGFD_ERR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  CGFD_ABI_END(h)
}

int cgfd_steps_done(const cgfd_solver *h, int *n) {
  CGFD_ABI_BEGIN
  if (!h || !n) return CGFD_ERR_ARG;
  *n = h->steps;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_get_seismograms(cgfd_solver *h, float *out, int *nt_done) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  if (nt_done) *nt_done = h->steps < h->d.nt ? h->steps : h->d.nt;
  if (h->nrecv && out)
    CK(h, cudaMemcpy(out, h->d_seis, (size_t)9 * h->nrecv * h->d.nt * sizeof(float),
                     cudaMemcpyDeviceToHost));
  return CGFD_OK;
  CGFD_ABI_END(h)
}

static void *set_ptr(cgfd_solver *h, int set, int comp) {
  if (comp < 0 || comp > 8) return nullptr;
  int s;
  if (set == CGFD_SET_FW) s = 0;
  else if (set == CGFD_SET_W) s = h->wcur;
  else if (set == CGFD_SET_TW) s = 3;
  else return nullptr;
  return (char *)h->set[s] + (size_t)comp * h->g.fstride * elem_size(h->elem);
}

int cgfd_get_field(cgfd_solver *h, int set, int comp, float *out) {
  CGFD_ABI_BEGIN
  if (!h || !out) return arg_fail(h, "null argument");
  void *p = set_ptr(h, set, comp);
  if (!p) return arg_fail(h, "bad set or component");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  const float sc = std::ldexp(1.f, h->sexp[comp]);
  int st = download_ref(h, p, out, h->elem, sc);
  if (st || set != CGFD_SET_TW || h->elem == ELEM_F32) return st;
  // 16-bit storage keeps tW - FW: add FW back
  std::vector<float> f(ref_n(h));
  st = download_ref(h, set_ptr(h, CGFD_SET_FW, comp), f.data(), h->elem, sc);
  if (st) return st;
  for (size_t t = 0; t < f.size(); ++t) out[t] += f[t];
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_set_field(cgfd_solver *h, int set, int comp, const float *in) {
  CGFD_ABI_BEGIN
  if (!h || !in) return arg_fail(h, "null argument");
  void *p = set_ptr(h, set, comp);
  if (!p) return arg_fail(h, "bad set or component");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  // only valid cells are taken; ghosts stay zero
  const long n = ref_n(h);
  const int nx = h->d.ni + 6, ny = h->d.nj + 6, nz = h->d.nk + 6;
  std::vector<float> v(n, 0.f);
  // 16-bit storage keeps tW - FW: subtract the stored FW
  std::vector<float> f;
  if (set == CGFD_SET_TW && h->elem != ELEM_F32) {
    f.resize(n);
    int st = download_ref(h, set_ptr(h, CGFD_SET_FW, comp), f.data(), h->elem,
                          std::ldexp(1.f, h->sexp[comp]));
    if (st) return st;
  }
  for (int i = LFD; i < nx - LFD; ++i)
    for (int j = LFD; j < ny - LFD; ++j)
      for (int k = LFD; k < nz - LFD; ++k) {
        const long t = ((long)i * ny + j) * nz + k;
        v[t] = f.empty() ? in[t] : in[t] - f[t];
      }
  return upload_ref(h, v.data(), p, h->elem, std::ldexp(1.f, -h->sexp[comp]));
  CGFD_ABI_END(h)
}

int cgfd_check_finite(cgfd_solver *h, long long *n_bad) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  DevGuard guard(h->d.device);
  if (h->elem == ELEM_F32)
    nonfinite_partial_kernel<<<h->nf_blocks, NF_THREADS, 0, h->st>>>(
        (const float *)h->set[0], 9 * h->g.fstride, h->d_partials);
  else
    nonfinite16_partial_kernel<<<h->nf_blocks, NF_THREADS, 0, h->st>>>(
        (const uint16_t *)h->set[0], 9 * h->g.fstride,
        (uint16_t)(h->elem == ELEM_F16 ? 0x7C00u : 0x7F80u), h->d_partials);
  CK(h, cudaGetLastError());
  nonfinite_sum_kernel<<<1, NF_THREADS, 0, h->st>>>(h->d_partials, h->nf_blocks);
  CK(h, cudaGetLastError());
  unsigned long long c = 0;
  CK(h, cudaMemcpyAsync(&c, h->d_partials + h->nf_blocks, sizeof(c), cudaMemcpyDeviceToHost,
                        h->st));
  CK(h, cudaStreamSynchronize(h->st));
  if (n_bad) *n_bad = (long long)c;
  if (c) {
    h->err = "non-finite values in the wavefield";
    return CGFD_ERR_NONFINITE;
  }
  return CGFD_OK;
  CGFD_ABI_END(h)
}


}  // extern "C"

// ------------------------- autotuning, batches -----------------------------

// Device state of a solver that a tuning run changes: the field sets, the
// ADE auxiliaries, the seismograms; saved before and put back after.
struct Snapshot {
  std::vector<std::pair<void *, size_t>> bufs;  // (device buffer, bytes)
  std::vector<void *> copies;
  int steps = 0;
};
static int snapshot_take(cgfd_solver *h, Snapshot &sn) {
  sn.bufs.clear();
  sn.bufs.push_back({h->state, 4 * 9 * h->g.fstride * elem_size(h->elem)});
  for (int d = 0; d < 3; ++d)
    if (h->aux[d])
      sn.bufs.push_back({h->aux[d], 3 * (size_t)h->g.ncaux * h->g.astride[d] * sizeof(float)});
  if (h->d_seis)
    sn.bufs.push_back({h->d_seis, (size_t)9 * h->nrecv * (h->d.nt > 0 ? h->d.nt : 1) * 4});
  sn.steps = h->steps;
  for (auto &b : sn.bufs) {
    void *c = nullptr;
    CK(h, cudaMalloc(&c, b.second));
    sn.copies.push_back(c);
    CK(h, cudaMemcpyAsync(c, b.first, b.second, cudaMemcpyDeviceToDevice, h->st));
  }
  CK(h, cudaStreamSynchronize(h->st));
  return CGFD_OK;
}
static int snapshot_restore(cgfd_solver *h, Snapshot &sn) {
  for (size_t q = 0; q < sn.bufs.size(); ++q)
    CK(h, cudaMemcpyAsync(sn.bufs[q].first, sn.copies[q], sn.bufs[q].second,
                          cudaMemcpyDeviceToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  for (void *c : sn.copies) cudaFree(c);
  sn.copies.clear();
  h->steps = sn.steps;
  return CGFD_OK;
}
// the work-list shapes the autotuner tries
// (the plan's current shape first, so the autotuner never ends on a worse
// one than it started from)
static std::vector<WorkParams> tuning_candidates(const WorkParams &current) {
  std::vector<WorkParams> v{current};
  for (int ipc : {3, 6, 12, 24})
    for (int mc : {12, 16, 24, 32, 48})
      for (double pw : {1.0, 2.0, 3.0}) {
        const WorkParams w{ipc, mc, pw};
        if (w.items_per_cta != current.items_per_cta || w.min_chunk != current.min_chunk ||
            w.pml_weight != current.pml_weight)
          v.push_back(w);
      }
  return v;
}

extern "C" {

int cgfd_autotune(cgfd_solver *h, int steps, float *best_ms) {
  CGFD_ABI_BEGIN
  if (!h || steps < 1) return arg_fail(h, "bad arguments");
  if (h->d.kernel != CGFD_KERNEL_FUSED) return arg_fail(h, "autotuning needs the default kernel");
  int st = cgfd_prepare(h);
  if (st) return st;
  DevGuard guard(h->d.device);
  Snapshot sn;
  st = snapshot_take(h, sn);
  if (st) return st;
  float best = 1e30f;
  WorkParams bestp = pair_get_work(h->plan);
  for (const WorkParams &wp : tuning_candidates(bestp)) {
    if (!pair_set_work(h->plan, wp)) continue;
    h->graphs_ok = false;
    st = build_graphs(h);
    if (st) break;
    h->steps = sn.steps;
    float ms = 0;
    st = cgfd_step(h, 1);  // warm-up
    if (!st) st = cgfd_step_timed(h, steps, &ms, nullptr);
    if (st) break;
    if (ms < best) { best = ms; bestp = wp; }
  }
  int st2 = snapshot_restore(h, sn);
  if (!st) st = st2;
  if (!pair_set_work(h->plan, bestp) && !st) st = cuda_fail(h, cudaErrorUnknown, "work list");
  h->graphs_ok = false;
  if (!st) st = build_graphs(h);
  if (best_ms) *best_ms = best / steps;
  return st;
  CGFD_ABI_END(h)
}

int cgfd_get_work_shape(cgfd_solver *h, int *items_per_cta, int *min_chunk, double *pml_weight) {
  CGFD_ABI_BEGIN
  if (!h || !items_per_cta || !min_chunk || !pml_weight) return arg_fail(h, "null argument");
  if (h->d.kernel != CGFD_KERNEL_FUSED || !h->plan)
    return arg_fail(h, "work shapes belong to the default kernel after cgfd_prepare");
  const WorkParams w = pair_get_work(h->plan);
  *items_per_cta = w.items_per_cta;
  *min_chunk = w.min_chunk;
  *pml_weight = w.pml_weight;
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_set_work_shape(cgfd_solver *h, int items_per_cta, int min_chunk, double pml_weight) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (h->d.kernel != CGFD_KERNEL_FUSED || !h->plan)
    return arg_fail(h, "work shapes belong to the default kernel after cgfd_prepare");
  if (items_per_cta < 1 || items_per_cta > 64 || min_chunk < 4 || min_chunk > 1024 ||
      !(pml_weight >= 0.0 && pml_weight <= 16.0))
    return arg_fail(h, "bad work shape");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  WorkParams w = pair_get_work(h->plan);
  w.items_per_cta = items_per_cta;
  w.min_chunk = min_chunk;
  w.pml_weight = pml_weight;
  if (!pair_set_work(h->plan, w)) return arg_fail(h, "work list rejected for this model");
  h->graphs_ok = false;  // the step graphs hold the launch configuration
  return build_graphs(h);
  CGFD_ABI_END(h)
}

int cgfd_test_withhold_copy(cgfd_solver *h, double wait_limit_s, int withhold) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (h->d.kernel != CGFD_KERNEL_FUSED || !h->plan)
    return arg_fail(h, "the wait test needs the default kernel");
  if (!(wait_limit_s > 0.0) || wait_limit_s > 60.0) return arg_fail(h, "wait limit out of range");
  if (!pair_set_wait_test(h->plan, wait_limit_s, withhold))
    return arg_fail(h, "wait test rejected");
  // the step graphs hold the kernels' parameters by value
  h->graphs_ok = false;
  if (!h->prepared) return CGFD_OK;  // cgfd_prepare builds them
  DevGuard guard(h->d.device);
  return build_graphs(h);
  CGFD_ABI_END(h)
}

}  // extern "C"

struct cgfd_batch {
  std::vector<cgfd_solver *> m;
  int device = 0;
  int elem = ELEM_F32;           // the members' storage type
  cudaStream_t st = nullptr;
  void *plan = nullptr;
  int *d_err = nullptr;
  SourceArgs *d_src = nullptr;   // [stage][model]
  RecordArgs *d_rec = nullptr;   // [model]
  bool any_src = false;
  int max_foc = 0;  // most focal points of any member
  int max_sp = 0;   // longest spread list (smoothed sources) of any member
  cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
  // launch shape: false, one persistent launch per stage part over every
  // member's items (uneven, small members share the GPU without tails);
  // true, every member's own step graphs on its own stream (members large
  // enough to fill the GPU alone run the single-model kernels, whose stage
  // arguments are kernel parameters).  cgfd_batch_autotune times both.
  bool member_launch = false;
  cudaEvent_t ev = nullptr;      // orders the batch's and the members' streams
  bool ready = false;
  int steps = 0;
  std::string err;
};

int cgfd::abi_exception(const cgfd_batch *b, const char *fn) noexcept {
  char buf[320];
  exception_text(fn, buf, sizeof(buf));
  try {
    if (b) const_cast<cgfd_batch *>(b)->err = buf;
    else g_last_create_error = buf;
  } catch (...) {
  }
  return CGFD_ERR_NOMEM;
}

static int batch_fail(cgfd_batch *b, int code, const std::string &msg) {
  if (b) b->err = msg;
  set_global_error(msg.c_str());
  return code;
}
#define BCK(b, call)                                                                  \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return batch_fail((b), CGFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static void batch_free(cgfd_batch *b) {
  for (auto &g : b->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (b->plan) { pair_destroy_plan(b->plan); b->plan = nullptr; }
  cudaFree(b->d_err);
  cudaFree(b->d_src);
  cudaFree(b->d_rec);
  b->d_err = nullptr; b->d_src = nullptr; b->d_rec = nullptr;
  if (b->ev) { cudaEventDestroy(b->ev); b->ev = nullptr; }
  if (b->st) { cudaStreamDestroy(b->st); b->st = nullptr; }
}

// the batched step of pattern p: per stage one launch per part over every
// model, the traction image, the sources; then the receiver record
template <typename T>
static void batch_sources(cgfd_batch *b, int rk) {
  const int n = (int)b->m.size();
  if (b->any_src)
    inject_sources_batch_kernel<T><<<n, 32, 0, b->st>>>(b->d_src + (size_t)rk * n);
  if (b->max_foc > 0)  // after the point sources (both may touch a cell)
    inject_focal_batch_kernel<T><<<dim3(focal_blocks(b->max_foc), n), 128, 0, b->st>>>(
        b->d_src + (size_t)rk * n);
  if (b->max_sp > 0)  // the smoothed sources last
    inject_spread_batch_kernel<T><<<dim3(spread_blocks(b->max_sp), n), 128, 0, b->st>>>(
        b->d_src + (size_t)rk * n);
}

static int batch_enqueue(cgfd_batch *b, int p, const std::vector<StageArgs> &args) {
  const int n = (int)b->m.size();
  for (int rk = 0; rk < 4; ++rk) {
    launch_stage_pair_batch(b->plan, p, args[(size_t)(p * 4 + rk) * n], b->d_err, b->st);
    BCK(b, cudaGetLastError());
    if (b->elem == ELEM_F16) batch_sources<__half>(b, rk);
    else if (b->elem == ELEM_BF16) batch_sources<__nv_bfloat16>(b, rk);
    else batch_sources<float>(b, rk);
    BCK(b, cudaGetLastError());
  }
  // the learned layers of the members that have one, after the step
  for (cgfd_solver *h : b->m)
    if (h->mlp_n) launch_mlp(h, b->st);
  BCK(b, cudaGetLastError());
  if (b->elem == ELEM_F16) record_batch_kernel<__half><<<n, 256, 0, b->st>>>(b->d_rec);
  else if (b->elem == ELEM_BF16) record_batch_kernel<__nv_bfloat16><<<n, 256, 0, b->st>>>(b->d_rec);
  else record_batch_kernel<float><<<n, 256, 0, b->st>>>(b->d_rec);
  BCK(b, cudaGetLastError());
  return CGFD_OK;
}

static int batch_build(cgfd_batch *b) {
  const int n = (int)b->m.size();
  static const int ins[4] = {0, 1, 2, 1}, outs[4] = {1, 2, 1, 0};
  std::vector<StageArgs> args((size_t)16 * n);
  std::vector<SourceArgs> src((size_t)4 * n);
  std::vector<RecordArgs> rec(n);
  b->any_src = false;
  b->max_foc = 0;
  b->max_sp = 0;
  for (int i = 0; i < n; ++i) {
    cgfd_solver *h = b->m[i];
    for (int p = 0; p < 4; ++p)
      for (int rk = 0; rk < 4; ++rk) {
        const int *dd = DIRS[p][rk];
        StageArgs &a = args[(size_t)(p * 4 + rk) * n + i];
        a = stage_args(h, rk, dd[0], dd[1], dd[2], ins[rk], outs[rk]);
        a.tw_skip = true;  // the batched paired kernels run with tW elision
      }
    for (int rk = 0; rk < 4; ++rk)
      src[(size_t)rk * n + i] = source_args(h, args[(size_t)rk * n + i], -1);
    if (h->nmnt + h->nfrc > 0) b->any_src = true;
    if (h->nfoc > b->max_foc) b->max_foc = h->nfoc;
    if (h->sp_n > b->max_sp) b->max_sp = h->sp_n;
    RecordArgs &r = rec[i];
    r.fw = h->set[0];
    r.fstride = h->g.fstride;
    r.cells = h->d_rcell;
    r.nrecv = h->nrecv;
    r.nt = h->d.nt;
    r.seis = h->d_seis;
    r.step = h->d_step;
    r.s = field_scales(h);
  }
  if (!b->plan) {
    std::vector<Geom> gs(n);
    std::vector<void *> sets((size_t)4 * n);
    std::vector<const float *> media(n), metric(n);
    std::vector<float *> aux((size_t)3 * n);
    for (int i = 0; i < n; ++i) {
      cgfd_solver *h = b->m[i];
      gs[i] = h->g;
      for (int q = 0; q < 4; ++q) sets[(size_t)4 * i + q] = h->set[q];
      media[i] = h->media;
      metric[i] = h->metric;
      for (int d = 0; d < 3; ++d) aux[(size_t)3 * i + d] = h->aux[d];
    }
    b->plan = pair_create_batch_plan(n, gs.data(), sets.data(), media.data(), metric.data(),
                                     aux.data(), b->elem);
    if (!b->plan) return batch_fail(b, CGFD_ERR_CUDA, "batch plan (tensor maps or work list)");
  }
  if (!pair_batch_set_args(b->plan, args.data()))
    return batch_fail(b, CGFD_ERR_CUDA, "batch stage arguments");
  if (!b->d_src) BCK(b, cudaMalloc(&b->d_src, src.size() * sizeof(SourceArgs)));
  if (!b->d_rec) BCK(b, cudaMalloc(&b->d_rec, rec.size() * sizeof(RecordArgs)));
  BCK(b, cudaMemcpy(b->d_src, src.data(), src.size() * sizeof(SourceArgs),
                    cudaMemcpyHostToDevice));
  BCK(b, cudaMemcpy(b->d_rec, rec.data(), rec.size() * sizeof(RecordArgs),
                    cudaMemcpyHostToDevice));
  for (int p = 0; p < 4; ++p) {
    if (b->graph[p]) { cudaGraphExecDestroy(b->graph[p]); b->graph[p] = nullptr; }
    cudaGraph_t gr = nullptr;
    BCK(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    int st = batch_enqueue(b, p, args);
    cudaError_t e = cudaStreamEndCapture(b->st, &gr);
    if (st) { if (gr) cudaGraphDestroy(gr); return st; }
    BCK(b, e);
    e = cudaGraphInstantiate(&b->graph[p], gr, 0);
    cudaGraphDestroy(gr);
    BCK(b, e);
  }
  b->ready = true;
  return CGFD_OK;
}

extern "C" {

int cgfd_batch_create(const cgfd_desc *descs, int n, cgfd_batch **out) {
  CGFD_ABI_BEGIN
  if (!descs || !out || n < 1) return batch_fail(nullptr, CGFD_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (descs[i].storage != descs[0].storage)
      return batch_fail(nullptr, CGFD_ERR_ARG, "batched models share one storage type");
    if (descs[i].kernel != CGFD_KERNEL_FUSED)
      return batch_fail(nullptr, CGFD_ERR_ARG, "batched models use the default kernel family");
    if (descs[i].device != descs[0].device)
      return batch_fail(nullptr, CGFD_ERR_ARG, "batched models share one device");
  }
  cgfd_batch *b = new cgfd_batch();
  b->device = descs[0].device;
  b->elem = descs[0].storage == CGFD_STORE_F16    ? ELEM_F16
            : descs[0].storage == CGFD_STORE_BF16 ? ELEM_BF16
                                                  : ELEM_F32;
  for (int i = 0; i < n; ++i) {
    cgfd_solver *h = nullptr;
    int st = cgfd_create(&descs[i], &h);
    if (st) {
      for (cgfd_solver *x : b->m) cgfd_destroy(x);
      delete b;
      return st;
    }
    b->m.push_back(h);
  }
  DevGuard guard(b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
  if (e != cudaSuccess) {
    batch_free(b);
    for (cgfd_solver *x : b->m) cgfd_destroy(x);
    delete b;
    return batch_fail(nullptr, CGFD_ERR_CUDA, "batch setup");
  }
  *out = b;
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

int cgfd_batch_solver(cgfd_batch *b, int i, cgfd_solver **h) {
  CGFD_ABI_BEGIN
  if (!b || !h || i < 0 || i >= (int)b->m.size())
    return batch_fail(b, CGFD_ERR_ARG, "bad model index");
  *h = b->m[i];
  b->ready = false;  // the caller may upload new inputs through it
  return CGFD_OK;
  CGFD_ABI_END(b)
}

int cgfd_batch_prepare(cgfd_batch *b) {
  CGFD_ABI_BEGIN
  if (!b) return batch_fail(b, CGFD_ERR_ARG, "null handle");
  for (cgfd_solver *h : b->m) {
    if (!h->prepared || !h->graphs_ok) b->ready = false;
    int st = cgfd_prepare(h);
    if (st) return batch_fail(b, st, h->err);
    if (h->steps != b->m[0]->steps)
      return batch_fail(b, CGFD_ERR_STATE, "batched models must be at the same step");
  }
  if (b->ready) return CGFD_OK;
  DevGuard guard(b->device);
  return batch_build(b);
  CGFD_ABI_END(b)
}

int cgfd_batch_step(cgfd_batch *b, int n_steps) {
  CGFD_ABI_BEGIN
  if (!b || n_steps < 0) return batch_fail(b, CGFD_ERR_ARG, "bad arguments");
  int st = cgfd_batch_prepare(b);
  if (st) return st;
  DevGuard guard(b->device);
  for (cgfd_solver *h : b->m) {
    const int last = h->steps + n_steps - 1;
    if (n_steps > 0 && h->nrecv && last >= h->d.nt)
      return batch_fail(b, CGFD_ERR_ARG, "more steps than a model's seismogram buffer (nt)");
    if (n_steps > 0 && ((h->nmnt && 2 * last + 2 >= h->nstfm) ||
                        (h->nfrc && 2 * last + 2 >= h->nstff)))
      return batch_fail(b, CGFD_ERR_ARG, "a model's source time function is too short");
    BCK(b, cudaMemcpyAsync(h->d_step, &h->steps, sizeof(int), cudaMemcpyHostToDevice, b->st));
  }
  // the batch's stream follows the work queued on the members' streams, and
  // the members' streams (seismograms, fields) follow the batch
  for (cgfd_solver *h : b->m) {
    BCK(b, cudaEventRecord(b->ev, h->st));
    BCK(b, cudaStreamWaitEvent(b->st, b->ev, 0));
  }
  if (b->member_launch) {
    // each member's own step graphs on its stream (the members' step counters
    // were set above, ordered on the batch's stream, which they now follow)
    BCK(b, cudaEventRecord(b->ev, b->st));
    for (cgfd_solver *h : b->m) {
      BCK(b, cudaStreamWaitEvent(h->st, b->ev, 0));
      for (int s = 0; s < n_steps; ++s)
        BCK(b, cudaGraphLaunch(h->graph[(h->steps + s) % 4], h->st));
    }
    // the batch's stream follows every member's last step
    for (cgfd_solver *h : b->m) {
      BCK(b, cudaEventRecord(b->ev, h->st));
      BCK(b, cudaStreamWaitEvent(b->st, b->ev, 0));
      h->steps += n_steps;
      h->wcur = 0;
    }
    return CGFD_OK;
  }
  const int s0 = b->m[0]->steps;
  for (int s = 0; s < n_steps; ++s) BCK(b, cudaGraphLaunch(b->graph[(s0 + s) % 4], b->st));
  BCK(b, cudaEventRecord(b->ev, b->st));
  for (cgfd_solver *h : b->m) {
    BCK(b, cudaStreamWaitEvent(h->st, b->ev, 0));
    h->steps += n_steps;
    h->wcur = 0;
  }
  return CGFD_OK;
  CGFD_ABI_END(b)
}

int cgfd_batch_sync(cgfd_batch *b, double timeout_s) {
  CGFD_ABI_BEGIN
  if (!b) return batch_fail(b, CGFD_ERR_ARG, "null handle");
  DevGuard guard(b->device);
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(b->st);
    if (e == cudaSuccess) {
      int flag = 0;
      BCK(b, cudaMemcpy(&flag, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
      for (cgfd_solver *h : b->m) {  // member launches record into the members' flags
        int f = 0;
        if (flag || !h->d_err) break;
        BCK(b, cudaMemcpy(&f, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        flag = f;
      }
      if (flag)
        return batch_fail(b, flag == 2 ? CGFD_ERR_CUDA : CGFD_ERR_TIMEOUT,
                          flag == 2 ? "stage kernel alignment self-check failed"
                                    : "a bounded wait inside a stage kernel expired");
      return CGFD_OK;
    }
    if (e != cudaErrorNotReady) BCK(b, e);
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (timeout_s >= 0 && el > timeout_s)
      return batch_fail(b, CGFD_ERR_TIMEOUT, "timeout waiting for the device");
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  CGFD_ABI_END(b)
}

int cgfd_batch_step_timed(cgfd_batch *b, int n_steps, float *ms) {
  CGFD_ABI_BEGIN
  if (!b || n_steps < 1 || !ms) return batch_fail(b, CGFD_ERR_ARG, "bad arguments");
  int st = cgfd_batch_prepare(b);
  if (st) return st;
  DevGuard guard(b->device);
  cudaEvent_t e0, e1;
  BCK(b, cudaEventCreate(&e0));
  BCK(b, cudaEventCreate(&e1));
  BCK(b, cudaEventRecord(e0, b->st));
  st = cgfd_batch_step(b, n_steps);
  if (st) return st;
  BCK(b, cudaEventRecord(e1, b->st));
  st = cgfd_batch_sync(b, -1);
  if (st) return st;
  BCK(b, cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return CGFD_OK;
  CGFD_ABI_END(b)
}

int cgfd_batch_autotune(cgfd_batch *b, int steps, float *best_ms) {
  CGFD_ABI_BEGIN
  if (!b || steps < 1) return batch_fail(b, CGFD_ERR_ARG, "bad arguments");
  int st = cgfd_batch_prepare(b);
  if (st) return st;
  DevGuard guard(b->device);
  std::vector<Snapshot> sn(b->m.size());
  for (size_t i = 0; i < b->m.size(); ++i) {
    st = snapshot_take(b->m[i], sn[i]);
    if (st) return batch_fail(b, st, b->m[i]->err);
  }
  float best = 1e30f;
  WorkParams bestp = pair_get_work(b->plan);
  for (const WorkParams &wp : tuning_candidates(bestp)) {
    if (!pair_set_work(b->plan, wp)) continue;
    b->ready = false;
    st = batch_build(b);
    if (st) break;
    for (size_t i = 0; i < b->m.size(); ++i) b->m[i]->steps = sn[i].steps;
    float ms = 0;
    st = cgfd_batch_step(b, 1);  // warm-up
    if (!st) st = cgfd_batch_step_timed(b, steps, &ms);
    if (st) break;
    if (ms < best) { best = ms; bestp = wp; }
  }
  // the other launch shape: every member's own step graphs, each with its
  // own work shape tuned first (cgfd_autotune restores the member's state)
  bool members_best = false;
  if (!st) {
    b->member_launch = true;
    for (size_t i = 0; i < b->m.size() && !st; ++i) {
      b->m[i]->steps = sn[i].steps;
      float member_ms = 0;
      st = cgfd_autotune(b->m[i], steps, &member_ms);
      if (st) st = batch_fail(b, st, b->m[i]->err);
    }
    for (size_t i = 0; i < b->m.size(); ++i) b->m[i]->steps = sn[i].steps;
    float ms = 0;
    st = cgfd_batch_step(b, 1);  // warm-up
    if (!st) st = cgfd_batch_step_timed(b, steps, &ms);
    if (!st && ms < best) { best = ms; members_best = true; }
    b->member_launch = false;
  }
  for (size_t i = 0; i < b->m.size(); ++i) {
    int st2 = snapshot_restore(b->m[i], sn[i]);
    if (!st) st = st2;
  }
  b->member_launch = members_best;
  if (!pair_set_work(b->plan, bestp) && !st) st = batch_fail(b, CGFD_ERR_CUDA, "work list");
  b->ready = false;
  if (!st) st = batch_build(b);
  if (best_ms) *best_ms = best / steps;
  return st;
  CGFD_ABI_END(b)
}

int cgfd_batch_set_launch(cgfd_batch *b, int shape) {
  CGFD_ABI_BEGIN
  if (!b || (shape != CGFD_BATCH_PERSISTENT && shape != CGFD_BATCH_MEMBERS))
    return batch_fail(b, CGFD_ERR_ARG, "bad launch shape");
  b->member_launch = shape == CGFD_BATCH_MEMBERS;
  return CGFD_OK;
  CGFD_ABI_END(b)
}

int cgfd_batch_get_launch(cgfd_batch *b, int *shape) {
  CGFD_ABI_BEGIN
  if (!b || !shape) return batch_fail(b, CGFD_ERR_ARG, "null argument");
  *shape = b->member_launch ? CGFD_BATCH_MEMBERS : CGFD_BATCH_PERSISTENT;
  return CGFD_OK;
  CGFD_ABI_END(b)
}

int cgfd_batch_last_error(cgfd_batch *b, char *buf, size_t len) {
  CGFD_ABI_BEGIN
  if (!buf || len == 0) return CGFD_ERR_ARG;
  const std::string &m = b ? b->err : std::string();
  std::snprintf(buf, len, "%s", m.c_str());
  return CGFD_OK;
  CGFD_ABI_END(b)
}

int cgfd_batch_destroy(cgfd_batch *b) {
  CGFD_ABI_BEGIN
  if (!b) return CGFD_OK;
  {
    DevGuard guard(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    batch_free(b);
  }
  for (cgfd_solver *h : b->m) cgfd_destroy(h);
  delete b;
  return CGFD_OK;
  CGFD_ABI_END(b)
}


// ------------------------------- outputs -----------------------------------

int cgfd_enable_peak_velocity(cgfd_solver *h, int on) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  if (on) {
    if (!h->d_pgv) CK(h, cudaMalloc(&h->d_pgv, 3 * h->g.plane * sizeof(float)));
    CK(h, cudaMemset(h->d_pgv, 0, 3 * h->g.plane * sizeof(float)));
  } else if (h->d_pgv) {
    cudaFree(h->d_pgv);
    h->d_pgv = nullptr;
  }
  invalidate(h);  // the step graphs gain or lose the update
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_get_peak_velocity(cgfd_solver *h, float *out) {
  CGFD_ABI_BEGIN
  if (!h || !out) return arg_fail(h, "null argument");
  if (!h->d_pgv) {
    h->err = "peak velocity is not enabled";
    return CGFD_ERR_STATE;
  }
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  std::vector<float> v(3 * h->g.plane);
  CK(h, cudaMemcpy(v.data(), h->d_pgv, v.size() * sizeof(float), cudaMemcpyDeviceToHost));
  const int ni = h->d.ni, nj = h->d.nj;
  for (int q = 0; q < 3; ++q)
    for (int i = 0; i < ni; ++i)
      for (int j = 0; j < nj; ++j)
        out[((size_t)q * ni + i) * nj + j] =
            v[(size_t)q * h->g.plane + (size_t)(j + LFD) * h->g.px + i + XO];
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_get_snapshot(cgfd_solver *h, int set, const int *start, const int *count,
                      const int *stride, int comp_mask, float *out) {
  CGFD_ABI_BEGIN
  if (!h || !start || !count || !stride || !out) return arg_fail(h, "null argument");
  if (comp_mask <= 0 || comp_mask >= (1 << NCOMP)) return arg_fail(h, "bad component mask");
  const int n3[3] = {h->d.ni + 6, h->d.nj + 6, h->d.nk + 6};
  for (int a = 0; a < 3; ++a) {
    if (count[a] < 1 || stride[a] < 1 || start[a] < 0 ||
        start[a] + (long)(count[a] - 1) * stride[a] >= n3[a])
      return arg_fail(h, "snapshot outside the grid");
  }
  void *base = set_ptr(h, set, 0);
  if (!base) return arg_fail(h, "bad set");
  int nc = 0;
  for (int c = 0; c < NCOMP; ++c) nc += (comp_mask >> c) & 1;
  const size_t n = (size_t)nc * count[0] * count[1] * count[2];
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  // 16-bit storage keeps tW - FW: gather FW too and add it back
  const bool add_fw = set == CGFD_SET_TW && h->elem != ELEM_F32;
  const int parts = add_fw ? 2 : 1;
  float *tmp = nullptr;
  CK(h, cudaMalloc(&tmp, parts * n * sizeof(float)));
  ScaleSet sc;
  for (int c = 0; c < NCOMP; ++c) sc.sc[c] = std::ldexp(1.f, h->sexp[c]);
  const int3 st3 = make_int3(start[0], start[1], start[2]);
  const int3 cn3 = make_int3(count[0], count[1], count[2]);
  const int3 sd3 = make_int3(stride[0], stride[1], stride[2]);
  for (int q = 0; q < parts; ++q) {
    const void *src = q == 0 ? base : set_ptr(h, CGFD_SET_FW, 0);
    float *dst = tmp + (size_t)q * n;
    if (h->elem == ELEM_F16)
      snapshot_kernel<<<592, 256, 0, h->st>>>((const __half *)src, h->g, comp_mask, st3, cn3,
                                              sd3, sc, dst);
    else if (h->elem == ELEM_BF16)
      snapshot_kernel<<<592, 256, 0, h->st>>>((const __nv_bfloat16 *)src, h->g, comp_mask, st3,
                                              cn3, sd3, sc, dst);
    else
      snapshot_kernel<<<592, 256, 0, h->st>>>((const float *)src, h->g, comp_mask, st3, cn3, sd3,
                                              sc, dst);
  }
  std::vector<float> fw(add_fw ? n : 0);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, tmp, n * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess && add_fw)
    e = cudaMemcpyAsync(fw.data(), tmp + n, n * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  if (e != cudaSuccess) return cuda_fail(h, e, "snapshot");
  for (size_t t = 0; t < fw.size(); ++t) out[t] += fw[t];
  return CGFD_OK;
  CGFD_ABI_END(h)
}

// seismo.nc of the reference (src/seisnc.cpp:1229-1364) in NetCDF classic:
// TimeNum (record) x PointNum; Vx..Tyz, currTime = (it+1)*stept, Pnum, Lnum,
// posx/posy/posz
int cgfd_write_seismograms_nc(cgfd_solver *h, const char *path, const float *pos) {
  CGFD_ABI_BEGIN
  if (!h || !path) return arg_fail(h, "null argument");
  const int n = h->nrecv, nt = h->d.nt;
  int done = 0;
  std::vector<float> seis((size_t)9 * n * (nt > 0 ? nt : 1));
  int st = cgfd_get_seismograms(h, n ? seis.data() : nullptr, &done);
  if (st) return st;
  // [c][recv][t] -> per component [t][recv]
  std::vector<std::vector<float>> comp(9, std::vector<float>((size_t)done * n));
  for (int c = 0; c < 9; ++c)
    for (int r = 0; r < n; ++r)
      for (int t = 0; t < done; ++t)
        comp[c][(size_t)t * n + r] = seis[((size_t)c * n + r) * nt + t];
  std::vector<float> tcur(done);
  for (int t = 0; t < done; ++t) tcur[t] = (float)((t + 1) * h->d.stept);
  std::vector<int> pnum(n), lnum(n, 1);
  std::vector<float> px(n), py(n), pz(n);
  std::vector<int> rloc;
  for (int r = 0; r < n; ++r) {
    pnum[r] = r + 1;
    px[r] = pos ? pos[3 * r] : 0.f;
    py[r] = pos ? pos[3 * r + 1] : 0.f;
    pz[r] = pos ? pos[3 * r + 2] : 0.f;
  }
  using namespace nc;
  std::vector<Dim> dims = {{"TimeNum", 0}, {"PointNum", (size_t)n}};
  static const char *names[9] = {"Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Txy", "Txz", "Tyz"};
  std::vector<Var> vars;
  for (int c = 0; c < 9; ++c) vars.push_back({names[c], NC_FLOAT, {0, 1}, comp[c].data()});
  vars.push_back({"currTime", NC_FLOAT, {0}, tcur.data()});
  vars.push_back({"Pnum", NC_INT, {1}, pnum.data()});
  vars.push_back({"Lnum", NC_INT, {1}, lnum.data()});
  vars.push_back({"posx", NC_FLOAT, {1}, px.data()});
  vars.push_back({"posy", NC_FLOAT, {1}, py.data()});
  vars.push_back({"posz", NC_FLOAT, {1}, pz.data()});
  const std::string content("Velocity and Stress seismogram", 31);  // with its NUL, as written
  if (!write_classic(path, dims, {{"Content", content}}, vars, (size_t)done)) {
    h->err = std::string("cannot write ") + path;
    return CGFD_ERR_ARG;
  }
  return CGFD_OK;
  CGFD_ABI_END(h)
}

// peakvel.nc of the reference (src/seisnc.cpp:1671-1757) in NetCDF classic:
// i x j; Vx, Vy, Vz (the reference's file holds Vy in its Vz variable; this
// one holds Vz)
int cgfd_write_peak_velocity_nc(cgfd_solver *h, const char *path) {
  CGFD_ABI_BEGIN
  if (!h || !path) return arg_fail(h, "null argument");
  std::vector<float> pv((size_t)3 * h->d.ni * h->d.nj);
  int st = cgfd_get_peak_velocity(h, pv.data());
  if (st) return st;
  using namespace nc;
  const size_t m = (size_t)h->d.ni * h->d.nj;
  std::vector<Dim> dims = {{"i", (size_t)h->d.ni}, {"j", (size_t)h->d.nj}};
  std::vector<Var> vars = {{"Vx", NC_FLOAT, {0, 1}, pv.data()},
                           {"Vy", NC_FLOAT, {0, 1}, pv.data() + m},
                           {"Vz", NC_FLOAT, {0, 1}, pv.data() + 2 * m}};
  if (!write_classic(path, dims, {}, vars, 0)) {
    h->err = std::string("cannot write ") + path;
    return CGFD_ERR_ARG;
  }
  return CGFD_OK;
  CGFD_ABI_END(h)
}


// ------------------------- learned absorbing layer -------------------------

int cgfd_set_boundary_mlp(cgfd_solver *h, int width, const void *weights_fp16) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  for (void **p : {(void **)&h->d_mlp_cells, &h->d_mlp_w, (void **)&h->d_mlp_delta,
                   (void **)&h->d_mlp_gain})
    if (*p) { cudaFree(*p); *p = nullptr; }
  h->mlp_n = 0;
  h->mlp_width = 0;
  h->mlp_ijk.clear();
  invalidate(h);
  if (!weights_fp16) return CGFD_OK;
  const int ni = h->d.ni, nj = h->d.nj, nk = h->d.nk;
  if (width < 1 || width > 16 || ni < width + 5 || nj < width + 5 || nk < width + 5)
    return arg_fail(h, "bad layer width for this grid");
  const int *nb = h->d.nabs;
  // nearest absorbing face of a valid cell within the layer: 0 x-, 1 x+,
  // 2 y-, 3 y+, 4 z- (bottom); -1 outside the layer
  int depth = 0;  // of the last cell face() placed in the layer
  auto face = [&](int i, int j, int k) {
    const int dist[5] = {nb[0] > 0 ? i : 1 << 30, nb[1] > 0 ? ni - 1 - i : 1 << 30,
                         nb[2] > 0 ? j : 1 << 30, nb[3] > 0 ? nj - 1 - j : 1 << 30,
                         nb[4] > 0 ? k : 1 << 30};
    int best = -1, bd = width;
    for (int f = 0; f < 5; ++f)
      if (dist[f] < bd) { bd = dist[f]; best = f; }
    depth = bd;
    return best;
  };
  const long step[5] = {1, -1, (long)h->g.px, -(long)h->g.px, (long)h->g.plane};
  // cells in the order of the field layout (x fastest): neighbouring cells of
  // the list are neighbours in memory, so the correction kernels' gathers of
  // 16 consecutive cells are coalesced
  std::vector<int4> cells;
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const int f = face(i, j, k);
        if (f < 0) continue;
        cells.push_back(
            make_int4((int)gidx(h->g, i + XO, j + LFD, k + LFD), (int)step[f], depth, 0));
        h->mlp_ijk.insert(h->mlp_ijk.end(), {i + LFD, j + LFD, k + LFD});
      }
  h->mlp_n = (int)cells.size();
  if (!h->mlp_n) return CGFD_OK;
  CK(h, cudaMalloc(&h->d_mlp_cells, cells.size() * sizeof(int4)));
  CK(h, cudaMemcpy(h->d_mlp_cells, cells.data(), cells.size() * sizeof(int4),
                   cudaMemcpyHostToDevice));
  mlp_set_attrs();
  CK(h, cudaMalloc(&h->d_mlp_w, CGFD_MLP_PARAMS * 2));
  CK(h, cudaMemcpy(h->d_mlp_w, weights_fp16, CGFD_MLP_PARAMS * 2, cudaMemcpyHostToDevice));
  CK(h, cudaMalloc(&h->d_mlp_delta, (size_t)9 * h->mlp_n * sizeof(float)));
  CK(h, cudaMalloc(&h->d_mlp_gain, (size_t)9 * width * sizeof(float)));
  h->mlp_width = width;
  return cgfd_set_boundary_mlp_gains(h, nullptr);
  CGFD_ABI_END(h)
}

int cgfd_set_boundary_mlp_gains(cgfd_solver *h, const float *gains) {
  CGFD_ABI_BEGIN
  if (!h) return arg_fail(h, "null handle");
  if (!h->mlp_n) return arg_fail(h, "no learned layer set");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  std::vector<float> g((size_t)9 * h->mlp_width, 1.f);
  if (gains) std::memcpy(g.data(), gains, g.size() * sizeof(float));
  for (float v : g)
    if (!std::isfinite(v)) return arg_fail(h, "non-finite gain");
  CK(h, cudaMemcpy(h->d_mlp_gain, g.data(), g.size() * sizeof(float), cudaMemcpyHostToDevice));
  invalidate(h);
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_boundary_mlp_cells(cgfd_solver *h, int *ijk, int *n) {
  CGFD_ABI_BEGIN
  if (!h || !n) return arg_fail(h, "null argument");
  const int cap = *n;
  *n = h->mlp_n;
  if (ijk && cap >= h->mlp_n)
    std::memcpy(ijk, h->mlp_ijk.data(), h->mlp_ijk.size() * sizeof(int));
  return CGFD_OK;
  CGFD_ABI_END(h)
}

int cgfd_boundary_mlp_features(cgfd_solver *h, float *x, float *scale, float *rho_vp) {
  CGFD_ABI_BEGIN
  if (!h || !x || !scale || !rho_vp) return arg_fail(h, "null argument");
  if (!h->mlp_n) return arg_fail(h, "no learned layer set");
  DevGuard guard(h->d.device);
  CK(h, cudaStreamSynchronize(h->st));
  const size_t n = h->mlp_n, fs = h->g.fstride;
  float *d = nullptr;
  CK(h, cudaMalloc(&d, n * (45 + 2) * sizeof(float)));
  launch_mlp_features(h->set[0], h->elem, fs, field_scales(h), h->media, h->media + 2 * fs,
                      h->d_mlp_cells,
                      h->mlp_n, d, d + n * 45, d + n * 46, h->st);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(x, d, n * 45 * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(scale, d + n * 45, n * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rho_vp, d + n * 46, n * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(h, e, "layer features");
  return CGFD_OK;
  CGFD_ABI_END(h)
}

}  // extern "C"
