// mlp.cu -- the learned thin absorbing layer: a small MLP that corrects the
// wavefield in a thin CFS-PML layer after every time step, and the kernels
// that train it.
//
// Layer: the valid cells within `width` cells of an absorbing face (the
// faces with a PML; never the free surface).  Each cell takes the inward
// normal of its nearest absorbing face (ties: x before y before z).
//
// Features of a cell: the 9 components of FW at the cell and the next 4
// cells along its inward normal (45 values), the stresses divided by the
// local P impedance rho*vp (velocity units), all divided by the largest of
// them in magnitude (the cell's scale; a cell whose features are all zero
// gets no correction).  MLP: 45 -> 64 -> 64 -> 9, SiLU after both hidden
// layers, weights stored as FP16, FP32 accumulation.  Output y: the
// correction of the cell's 9 components in the same normalised units,
// bounded as G*tanh(y/G) (G = 0.25: a cell moves by at most a quarter of its
// feature scale per step), so dFW[c] = G*tanh(y[c]/G) * scale * (c < 3 ? 1 :
// rho*vp), times a gain per (depth in the layer, component) that the host
// sets (default 1).  Then each component's correction d_c (normalised
// units) is clamped so that it can only move the component toward zero:
// u_c + d_c lies between 0 and u_c (u: the cell's own 9 normalised values).
// The correction is thereby a state-dependent damping of the layer (a learned
// sponge on top of the PML): it never flips a sign nor grows a magnitude.  A
// correction that is homogeneous in the field and may add energy made long
// runs grow, and one bounded only in the cell's energy (which may still
// rotate energy between components) left a slowly growing late field.  The
// training target is the unbounded y.  The corrections of all layer cells
// are computed first and added in a second pass (a cell's features include
// other layer cells).
//
// Inference runs on the tensor cores: a warp takes 16 layer cells, stages
// their features in shared memory as FP16, and runs the three layers as
// mma.sync m16n8k16 (FP16 inputs, FP32 accumulation): layer 1 is 16x48
// (45 padded) times 48x64, layer 2 16x64 times 64x64, layer 3 16x64 times
// 64x16 (9 padded).  A layer's FP32 accumulators, after SiLU (once per
// hidden unit and cell), are the next layer's A operand in registers (the
// accumulator layout of m16n8 equals the A layout of k16 taken in pairs of
// n-tiles), so only the input features go through shared memory.  Field
// sets of any storage type (FP32, or FP16/BF16 with per-component scales).
//
// Training kernel: for samples (x, t) of normalised features and target
// corrections, the mean squared error over samples and its gradient with
// respect to every parameter.  A block takes chunks of 128 samples: one
// thread per sample runs the forward and backward pass (FP32) and leaves
// the inputs, activations and back-propagated errors in shared memory; then
// every thread sums, over the chunk's samples, the products for the
// parameters it owns (a block-level reduction, no atomics), carrying the
// sums across the block's chunks; per-block partial gradients are summed in
// block order by a second kernel, so the result does not depend on timing.
#include "../../include/cgfd.h"
#include "abi_guard.h"
#include "cgfd_internal.cuh"
#include "elem.cuh"

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

namespace cgfd {
namespace mlp {

constexpr int NIN = 45, NH = 64, NOUT = 9;
constexpr float MIN_SCALE = 1e-30f;  // smaller feature scales get no correction
constexpr float GAIN = 0.25f;        // corrections are G*tanh(y/G): |dFW| <= G*scale
// parameter offsets: W1 [NH][NIN], b1 [NH], W2 [NH][NH], b2 [NH], W3 [NOUT][NH], b3 [NOUT]
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH;
constexpr int OW3 = OB2 + NH, OB3 = OW3 + NOUT * NH, NPAR = OB3 + NOUT;
static_assert(NPAR == CGFD_MLP_PARAMS, "parameter count of the ABI");

__device__ __forceinline__ float silu(float a) { return a / (1.f + __expf(-a)); }
// the inference form: one fast reciprocal instead of an IEEE division (its
// relative error, a few units in the last FP32 place, is far below the FP16
// rounding of the activation that follows)
__device__ __forceinline__ float silu_fast(float a) { return __fdividef(a, 1.f + __expf(-a)); }
// d silu / da
__device__ __forceinline__ float dsilu(float a) {
  const float s = 1.f / (1.f + __expf(-a));
  return s * (1.f + a * (1.f - s));
}

// ------------------------------ inference ---------------------------------
// Shared memory of the inference kernel: the weights as FP16 rows [n][k]
// (the B operands), row strides padded so that a fragment's 32 loads hit 32
// banks; per warp a 16-cell tile of features.
constexpr int K1 = 48, LD1 = 56, LD2 = 72, NOP = 16;  // padded K, row strides, padded outputs
constexpr int LDX = 56;                               // feature tile row stride (halves)
struct WSmem {
  __half w1[NH * LD1];
  __half w2[NH * LD2];
  __half w3[NOP * LD2];
  float b1[NH], b2[NH], b3[NOP];
};
struct TileSmem {
  __half x[16 * LDX];  // normalised features of the 16 cells, FP16
  float own[16 * NOUT];  // the cells' own 9 normalised values (FP32)
  float scale[16], z[16];
  int depth[16];       // the cells' depths in the layer (gain rows)
};
constexpr int INF_WARPS = 4;
constexpr int MAX_WIDTH = 16;  // widest layer cgfd_set_boundary_mlp accepts
// weights, the gain table [MAX_WIDTH][NOUT] and the warps' tiles
constexpr size_t INF_SMEM =
    sizeof(WSmem) + MAX_WIDTH * NOUT * sizeof(float) + INF_WARPS * sizeof(TileSmem);

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t lds32(const __half *p) {
  return *reinterpret_cast<const uint32_t *>(p);
}
// D = A(16x16, row) * B(16x8, col) + C, FP16 inputs, FP32 accumulators
__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ void load_weights(const __half *w, WSmem &s) {
  const int t = threadIdx.x, nt = blockDim.x;
  for (int q = t; q < NH * LD1; q += nt) {
    const int n = q / LD1, k = q % LD1;
    s.w1[q] = k < NIN ? w[OW1 + n * NIN + k] : __float2half(0.f);
  }
  for (int q = t; q < NH * LD2; q += nt) {
    const int n = q / LD2, k = q % LD2;
    s.w2[q] = k < NH ? w[OW2 + n * NH + k] : __float2half(0.f);
  }
  for (int q = t; q < NOP * LD2; q += nt) {
    const int n = q / LD2, k = q % LD2;
    s.w3[q] = (n < NOUT && k < NH) ? w[OW3 + n * NH + k] : __float2half(0.f);
  }
  for (int q = t; q < NH; q += nt) {
    s.b1[q] = __half2float(w[OB1 + q]);
    s.b2[q] = __half2float(w[OB2 + q]);
  }
  for (int q = t; q < NOP; q += nt) s.b3[q] = q < NOUT ? __half2float(w[OB3 + q]) : 0.f;
  __syncthreads();
}

// The features of the warp's 16 cells (cells[q0 .. q0+15], fewer at the
// end) into the tile: lane & 15 is the cell, lanes 0-15 take stencil points
// 0-2 and lanes 16-31 points 3-4.  Every loop has a fixed trip count, so
// the lane's 27 (18) field loads are all issued before the first use and
// its values stay in registers.  A cell without a correction gets scale 0
// and zero features.
template <typename T>
__device__ __forceinline__ void stage_features(const T *fw, size_t fs, const float *sc,
                                               const float *lam2mu, const float *irho,
                                               const int4 *cells, int n, int q0, TileSmem &tl) {
  const int lane = threadIdx.x & 31, r = lane & 15, half = lane >> 4;
  const int q = q0 + r;
  const bool live = q < n;
  int4 cell = make_int4(0, 0, 0, 0);
  if (live) cell = cells[q];
  const int s0 = half ? 3 : 0, np = half ? 2 : 3;  // first stencil point, points taken
  float v[3][NOUT];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const bool on = live && k < np;
    const size_t o = on ? (size_t)((long)cell.x + (long)(s0 + k) * cell.y) : 0;
#pragma unroll
    for (int c = 0; c < NOUT; ++c) v[k][c] = on ? Elem<T>::ld(fw + (size_t)c * fs + o) : 0.f;
  }
  const float z = live ? sqrtf(lam2mu[cell.x] / irho[cell.x]) : 1.f;  // rho vp
  const float rz = 1.f / z;
  float m = 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < NOUT; ++c) {
      float x = v[k][c] * sc[c];
      if (c >= 3) x *= rz;
      v[k][c] = x;
      m = fmaxf(m, fabsf(x));
    }
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
  const bool on = live && m > MIN_SCALE;
  const float rinv = on ? 1.f / m : 0.f;
  __half *xr = tl.x + r * LDX + s0 * NOUT;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < NOUT; ++c) {
      const float x = v[k][c] * rinv;
      if (k < np) xr[k * NOUT + c] = __float2half_rn(x);
      if (k == 0 && !half) tl.own[r * NOUT + c] = x;
    }
  if (half) {
#pragma unroll
    for (int k = NIN; k < LDX; ++k) tl.x[r * LDX + k] = __float2half(0.f);
  } else {
    tl.scale[r] = on ? m : 0.f;
    tl.z[r] = z;
    tl.depth[r] = cell.z;
  }
}

// the MLP of the 16 cells of a tile: y (rows g and g+8, columns 2t, 2t+1
// of the two output n-tiles) in out[2][4] as the mma accumulators hold them
__device__ void mlp_tile(const WSmem &w, const TileSmem &tl, float (&out)[2][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // layer 1: [16 x 48] x [48 x 64]
  float acc[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = w.b1[nt * 8 + 2 * t], b1 = w.b1[nt * 8 + 2 * t + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
  }
#pragma unroll
  for (int ks = 0; ks < K1 / 16; ++ks) {
    const __half *xa = tl.x + g * LDX + ks * 16 + 2 * t;
    const uint32_t a0 = lds32(xa), a1 = lds32(xa + 8 * LDX);
    const uint32_t a2 = lds32(xa + 8), a3 = lds32(xa + 8 * LDX + 8);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __half *wb = w.w1 + (nt * 8 + g) * LD1 + ks * 16 + 2 * t;
      mma16816(acc[nt], a0, a1, a2, a3, lds32(wb), lds32(wb + 8));
    }
  }
  // SiLU, as FP16 A operands of layer 2 (n-tiles 2ks and 2ks+1 = k-step ks)
  uint32_t ha[4][4];
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    const float *c0 = acc[2 * ks], *c1 = acc[2 * ks + 1];
    ha[ks][0] = pack_h2(silu_fast(c0[0]), silu_fast(c0[1]));
    ha[ks][1] = pack_h2(silu_fast(c0[2]), silu_fast(c0[3]));
    ha[ks][2] = pack_h2(silu_fast(c1[0]), silu_fast(c1[1]));
    ha[ks][3] = pack_h2(silu_fast(c1[2]), silu_fast(c1[3]));
  }
  // layer 2: [16 x 64] x [64 x 64]
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = w.b2[nt * 8 + 2 * t], b1 = w.b2[nt * 8 + 2 * t + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
  }
#pragma unroll
  for (int ks = 0; ks < 4; ++ks)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __half *wb = w.w2 + (nt * 8 + g) * LD2 + ks * 16 + 2 * t;
      mma16816(acc[nt], ha[ks][0], ha[ks][1], ha[ks][2], ha[ks][3], lds32(wb), lds32(wb + 8));
    }
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    const float *c0 = acc[2 * ks], *c1 = acc[2 * ks + 1];
    ha[ks][0] = pack_h2(silu_fast(c0[0]), silu_fast(c0[1]));
    ha[ks][1] = pack_h2(silu_fast(c0[2]), silu_fast(c0[3]));
    ha[ks][2] = pack_h2(silu_fast(c1[0]), silu_fast(c1[1]));
    ha[ks][3] = pack_h2(silu_fast(c1[2]), silu_fast(c1[3]));
  }
  // layer 3: [16 x 64] x [64 x 16]
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    const float b0 = w.b3[nt * 8 + 2 * t], b1 = w.b3[nt * 8 + 2 * t + 1];
    out[nt][0] = b0; out[nt][1] = b1; out[nt][2] = b0; out[nt][3] = b1;
  }
#pragma unroll
  for (int ks = 0; ks < 4; ++ks)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      const __half *wb = w.w3 + (nt * 8 + g) * LD2 + ks * 16 + 2 * t;
      mma16816(out[nt], ha[ks][0], ha[ks][1], ha[ks][2], ha[ks][3], lds32(wb), lds32(wb + 8));
    }
}

// corrections of all layer cells into delta [9][n] (values, not stored units);
// gain: [width][9], width <= MAX_WIDTH
template <typename T>
__global__ void __launch_bounds__(INF_WARPS * 32)
    delta_kernel(const T *__restrict__ fw, size_t fs, ScaleSet scs, const float *lam2mu,
                 const float *irho, const int4 *__restrict__ cells, int n,
                 const __half *__restrict__ wts, const float *__restrict__ gain, int width,
                 float *__restrict__ delta) {
  extern __shared__ __align__(16) unsigned char smem[];
  WSmem &w = *reinterpret_cast<WSmem *>(smem);
  float *sgain = reinterpret_cast<float *>(smem + sizeof(WSmem));
  TileSmem &tl = reinterpret_cast<TileSmem *>(smem + sizeof(WSmem) +
                                               MAX_WIDTH * NOUT * sizeof(float))[threadIdx.x >> 5];
  for (int q = threadIdx.x; q < width * NOUT; q += blockDim.x) sgain[q] = gain[q];
  load_weights(wts, w);  // ends with a block barrier
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int warp = blockIdx.x * INF_WARPS + (threadIdx.x >> 5);
  const int nwarps = gridDim.x * INF_WARPS;
  for (int q0 = warp * 16; q0 < n; q0 += nwarps * 16) {
    stage_features<T>(fw, fs, scs.sc, lam2mu, irho, cells, n, q0, tl);
    __syncwarp();
    float y[2][4];
    mlp_tile(w, tl, y);
    // this thread's outputs: rows g, g+8; columns 2t, 2t+1 (+8 for n-tile 1)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = g + (e >> 1) * 8, c = nt * 8 + 2 * t + (e & 1);
        const int q = q0 + r;
        if (c >= NOUT || q >= n) continue;
        const float s = tl.scale[r];
        float d = 0.f;
        if (s > 0.f) {
          const float u = tl.own[r * NOUT + c];
          d = sgain[tl.depth[r] * NOUT + c] * GAIN * tanhf(y[nt][e] / GAIN);
          d = fminf(fmaxf(d, fminf(0.f, -u)), fmaxf(0.f, -u));
        }
        delta[(size_t)c * n + q] = d * s * (c < 3 ? 1.f : tl.z[r]);
      }
    __syncwarp();  // the tile is reused by the warp's next 16 cells
  }
}

// one thread per layer cell: its 9 components read first, then written
template <typename T>
__global__ void __launch_bounds__(256)
    apply_kernel(T *__restrict__ fw, size_t fs, ScaleSet scs, const int4 *__restrict__ cells,
                 int n, const float *__restrict__ delta) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  T *p = fw + (size_t)cells[q].x;
  float u[NOUT];
#pragma unroll
  for (int c = 0; c < NOUT; ++c)  // in stored units: the component's scale divides the correction
    u[c] = Elem<T>::ld(p + (size_t)c * fs) + delta[(size_t)c * n + q] / scs.sc[c];
#pragma unroll
  for (int c = 0; c < NOUT; ++c) Elem<T>::st(p + (size_t)c * fs, u[c]);
}

// normalised features and scales of all layer cells (training samples):
// the same features as the inference kernel, in FP32
template <typename T>
__global__ void features_kernel(const T *__restrict__ fw, size_t fs, ScaleSet scs,
                                const float *lam2mu, const float *irho,
                                const int4 *__restrict__ cells, int n, float *__restrict__ xs,
                                float *__restrict__ scales, float *__restrict__ zs) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int4 cell = cells[q];
    const float z = sqrtf(lam2mu[cell.x] / irho[cell.x]), rz = 1.f / z;
    float x[NIN], m = 0.f;
    for (int s = 0; s < 5; ++s)
      for (int c = 0; c < NOUT; ++c) {
        float v = Elem<T>::ld(fw + (size_t)c * fs + cell.x + (long)s * cell.y) * scs.sc[c];
        if (c >= 3) v *= rz;
        x[s * NOUT + c] = v;
        m = fmaxf(m, fabsf(v));
      }
    const bool on = m > MIN_SCALE;
    const float r = on ? 1.f / m : 0.f;
    for (int k = 0; k < NIN; ++k) xs[(size_t)q * NIN + k] = x[k] * r;
    scales[q] = on ? m : 0.f;
    zs[q] = z;
  }
}

// ------------------------------- training ---------------------------------
constexpr int GB = 128;       // samples per chunk = threads per block
constexpr int LDS = GB + 1;   // row stride of the per-chunk arrays (bank spread)
constexpr int PER_T = (NPAR + GB - 1) / GB;  // parameters owned per thread
// shared memory: FP32 parameters, then [row][sample] arrays of the chunk
constexpr int R_X = 0, R_H1 = R_X + NIN, R_H2 = R_H1 + NH, R_DY = R_H2 + NH;
constexpr int R_D2 = R_DY + NOUT, R_D1 = R_D2 + NH, NROWS = R_D1 + NH;
constexpr size_t GRAD_SMEM = (NPAR + (size_t)NROWS * LDS) * sizeof(float);

// the sum over the chunk of (row a) * (row b), or of row a (b < 0)
__device__ __forceinline__ float row_dot(const float *ch, int a, int b) {
  const float *pa = ch + a * LDS;
  float s = 0.f;
  if (b < 0) {
    for (int k = 0; k < GB; ++k) s += pa[k];
  } else {
    const float *pb = ch + b * LDS;
    for (int k = 0; k < GB; ++k) s = fmaf(pa[k], pb[k], s);
  }
  return s;
}
// rows whose product over samples is parameter p's gradient
__device__ __forceinline__ void param_rows(int p, int *a, int *b) {
  if (p < OB1) { *a = R_D1 + (p - OW1) / NIN; *b = R_X + (p - OW1) % NIN; }
  else if (p < OW2) { *a = R_D1 + (p - OB1); *b = -1; }
  else if (p < OB2) { *a = R_D2 + (p - OW2) / NH; *b = R_H1 + (p - OW2) % NH; }
  else if (p < OW3) { *a = R_D2 + (p - OB2); *b = -1; }
  else if (p < OB3) { *a = R_DY + (p - OW3) / NH; *b = R_H2 + (p - OW3) % NH; }
  else { *a = R_DY + (p - OB3); *b = -1; }
}

__global__ void __launch_bounds__(GB)
    grad_kernel(const __half *__restrict__ w, const float *__restrict__ xs,
                const float *__restrict__ ts, int n, float *__restrict__ partial) {
  extern __shared__ __align__(16) unsigned char gsm[];
  float *sw = reinterpret_cast<float *>(gsm);  // NPAR parameters (FP32)
  float *ch = sw + NPAR;                       // the chunk's rows
  for (int q = threadIdx.x; q < NPAR; q += GB) sw[q] = __half2float(w[q]);
  __syncthreads();
  const int s = threadIdx.x;
  const float inv_n = 1.f / (float)n;
  float acc[PER_T];
#pragma unroll
  for (int e = 0; e < PER_T; ++e) acc[e] = 0.f;
  float lsum = 0.f;
  for (int c0 = blockIdx.x * GB; c0 < n; c0 += gridDim.x * GB) {
    const int sample = c0 + s;
    const bool live = sample < n;
    // forward and backward of this thread's sample, into the chunk's rows
    for (int k = 0; k < NIN; ++k) ch[(R_X + k) * LDS + s] = live ? xs[(size_t)sample * NIN + k] : 0.f;
    for (int o = 0; o < NH; ++o) {
      float a = sw[OB1 + o];
      for (int k = 0; k < NIN; ++k) a = fmaf(sw[OW1 + o * NIN + k], ch[(R_X + k) * LDS + s], a);
      ch[(R_H1 + o) * LDS + s] = silu(a);
      ch[(R_D1 + o) * LDS + s] = dsilu(a);  // dL/da1 after the backward pass
    }
    for (int o = 0; o < NH; ++o) {
      float a = sw[OB2 + o];
      for (int k = 0; k < NH; ++k) a = fmaf(sw[OW2 + o * NH + k], ch[(R_H1 + k) * LDS + s], a);
      ch[(R_H2 + o) * LDS + s] = silu(a);
      ch[(R_D2 + o) * LDS + s] = dsilu(a);  // dL/da2 after the backward pass
    }
    for (int c = 0; c < NOUT; ++c) {
      float y = sw[OB3 + c];
      for (int k = 0; k < NH; ++k) y = fmaf(sw[OW3 + c * NH + k], ch[(R_H2 + k) * LDS + s], y);
      const float e = live ? y - ts[(size_t)sample * NOUT + c] : 0.f;
      lsum += e * e;
      ch[(R_DY + c) * LDS + s] = 2.f * e * inv_n;
    }
    for (int q = 0; q < NH; ++q) {  // dL/da2
      float d = 0.f;
      for (int c = 0; c < NOUT; ++c) d = fmaf(sw[OW3 + c * NH + q], ch[(R_DY + c) * LDS + s], d);
      ch[(R_D2 + q) * LDS + s] *= d;
    }
    for (int q = 0; q < NH; ++q) {  // dL/da1
      float d = 0.f;
      for (int o = 0; o < NH; ++o) d = fmaf(sw[OW2 + o * NH + q], ch[(R_D2 + o) * LDS + s], d);
      ch[(R_D1 + q) * LDS + s] *= d;
    }
    __syncthreads();
    // the chunk's contribution to this thread's parameters
#pragma unroll
    for (int e = 0; e < PER_T; ++e) {
      const int p = threadIdx.x + e * GB;
      if (p < NPAR) {
        int a, b;
        param_rows(p, &a, &b);
        acc[e] += row_dot(ch, a, b);
      }
    }
    __syncthreads();  // the rows are rewritten by the next chunk
  }
  float *out = partial + (size_t)blockIdx.x * (NPAR + 1);
#pragma unroll
  for (int e = 0; e < PER_T; ++e) {
    const int p = threadIdx.x + e * GB;
    if (p < NPAR) out[p] = acc[e];
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  __shared__ float lw[GB / 32];
  if ((threadIdx.x & 31) == 0) lw[threadIdx.x >> 5] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float l = 0.f;
    for (int q = 0; q < GB / 32; ++q) l += lw[q];
    out[NPAR] = l * inv_n;
  }
}

// sums the per-block partials in block order (deterministic)
__global__ void reduce_partials(const float *__restrict__ partial, int nblocks,
                                float *__restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= NPAR; p += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * (NPAR + 1) + p];
    out[p] = s;
  }
}

}  // namespace mlp

size_t mlp_delta_smem() { return mlp::INF_SMEM; }

namespace {
int mlp_blocks(int n) {
  const int b = (n + 127) / 128;
  return b < 1 ? 1 : (b < 592 ? b : 592);
}
template <typename T>
void mlp_step_t(const void *fw, size_t fs, const ScaleSet &sc, const float *lam2mu,
                const float *irho, const int4 *cells, int n, const void *w, const float *gain,
                int width, float *delta, cudaStream_t s) {
  // every 16 cells are one warp's tile
  int blocks = (n + 16 * mlp::INF_WARPS - 1) / (16 * mlp::INF_WARPS);
  blocks = blocks < 1 ? 1 : (blocks < 4 * 148 ? blocks : 4 * 148);
  mlp::delta_kernel<T><<<blocks, mlp::INF_WARPS * 32, mlp::INF_SMEM, s>>>(
      (const T *)fw, fs, sc, lam2mu, irho, cells, n, (const __half *)w, gain, width, delta);
  mlp::apply_kernel<T><<<(n + 255) / 256, 256, 0, s>>>((T *)const_cast<void *>(fw), fs, sc,
                                                       cells, n, delta);
}
}  // namespace

void mlp_set_attrs() {
  cudaFuncSetAttribute(mlp::delta_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mlp::INF_SMEM);
  cudaFuncSetAttribute(mlp::delta_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mlp::INF_SMEM);
  cudaFuncSetAttribute(mlp::delta_kernel<__nv_bfloat16>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::INF_SMEM);
}

void launch_mlp_step(const void *fw, int elem, size_t fs, const ScaleSet &sc, const float *lam2mu,
                     const float *irho, const int4 *cells, int n, const void *w, const float *gain,
                     int width, float *delta, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n <= 0 || width < 1 || width > mlp::MAX_WIDTH) return;  // the setter refuses such layers
  if (elem == ELEM_F16)
    mlp_step_t<__half>(fw, fs, sc, lam2mu, irho, cells, n, w, gain, width, delta, s);
  else if (elem == ELEM_BF16)
    mlp_step_t<__nv_bfloat16>(fw, fs, sc, lam2mu, irho, cells, n, w, gain, width, delta, s);
  else
    mlp_step_t<float>(fw, fs, sc, lam2mu, irho, cells, n, w, gain, width, delta, s);
}

void launch_mlp_features(const void *fw, int elem, size_t fs, const ScaleSet &sc,
                         const float *lam2mu, const float *irho, const int4 *cells, int n,
                         float *xs, float *scales, float *zs, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const int b = mlp_blocks(n);
  if (elem == ELEM_F16)
    mlp::features_kernel<__half><<<b, 128, 0, s>>>((const __half *)fw, fs, sc, lam2mu, irho,
                                                   cells, n, xs, scales, zs);
  else if (elem == ELEM_BF16)
    mlp::features_kernel<__nv_bfloat16><<<b, 128, 0, s>>>((const __nv_bfloat16 *)fw, fs, sc,
                                                          lam2mu, irho, cells, n, xs, scales, zs);
  else
    mlp::features_kernel<float><<<b, 128, 0, s>>>((const float *)fw, fs, sc, lam2mu, irho, cells,
                                                  n, xs, scales, zs);
}

}  // namespace cgfd

using namespace cgfd;

namespace {

// device buffers of cgfd_mlp_gradient, kept between calls (grown on demand)
// per device; calls are serialised by the mutex
struct GradBuffers {
  void *w = nullptr;
  float *x = nullptr, *t = nullptr, *partial = nullptr, *out = nullptr;
  size_t ncap = 0;
  int nblocks = 0;
};
std::mutex g_grad_lock;
std::vector<GradBuffers> g_grad;

}  // namespace

extern "C" int cgfd_mlp_gradient(const void *weights_fp16, const float *x, const float *t, int n,
                                 float *grad, float *loss) {
  CGFD_ABI_BEGIN
  if (!weights_fp16 || !x || !t || n < 1 || !grad || !loss) {
    set_global_error("cgfd_mlp_gradient: bad arguments");
    return CGFD_ERR_ARG;
  }
  using namespace cgfd::mlp;
  std::lock_guard<std::mutex> lk(g_grad_lock);
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    set_global_error(cudaGetErrorString(e));
    return CGFD_ERR_CUDA;
  }
  if ((int)g_grad.size() <= dev) g_grad.resize(dev + 1);
  GradBuffers &B = g_grad[dev];
  if (!B.w) {
    B.nblocks = sms > 0 ? sms : 148;
    e = cudaMalloc(&B.w, NPAR * sizeof(__half));
    if (e == cudaSuccess)
      e = cudaMalloc(&B.partial, (size_t)B.nblocks * (NPAR + 1) * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&B.out, (NPAR + 1) * sizeof(float));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)GRAD_SMEM);
  }
  if (e == cudaSuccess && (size_t)n > B.ncap) {
    cudaFree(B.x);
    cudaFree(B.t);
    B.x = B.t = nullptr;
    B.ncap = 0;
    e = cudaMalloc(&B.x, (size_t)n * NIN * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&B.t, (size_t)n * NOUT * sizeof(float));
    if (e == cudaSuccess) B.ncap = (size_t)n;
  }
  if (e == cudaSuccess) e = cudaMemcpy(B.w, weights_fp16, NPAR * sizeof(__half), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B.x, x, (size_t)n * NIN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B.t, t, (size_t)n * NOUT * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    int blocks = (n + GB - 1) / GB;
    if (blocks > B.nblocks) blocks = B.nblocks;
    grad_kernel<<<blocks, GB, GRAD_SMEM>>>((const __half *)B.w, B.x, B.t, n, B.partial);
    reduce_partials<<<(NPAR + 256) / 256, 256>>>(B.partial, blocks, B.out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(grad, B.out, NPAR * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(loss, B.out + NPAR, sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    set_global_error(cudaGetErrorString(e));
    return CGFD_ERR_CUDA;
  }
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}
