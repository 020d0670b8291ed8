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
// layers, weights and biases stored as FP16, arithmetic in FP32.  Output y:
// the correction of the cell's 9 components in the same normalised units,
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
// training target is the unbounded y.
// The corrections of all
// layer cells are computed first and added in a second pass (a cell's
// features include other layer cells).
//
// Training kernel: for samples (x, t) of normalised features and target
// corrections, the mean squared error over samples and its gradient with
// respect to every parameter (backpropagation written out per layer).
#include "../../include/cgfd.h"
#include "cgfd_internal.cuh"

#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace cgfd {
namespace mlp {

constexpr int NIN = 45, NH = 64, NOUT = 9;
constexpr float MIN_SCALE = 1e-30f;  // smaller feature scales get no correction
constexpr float GAIN = 0.25f;        // corrections are G*tanh(y/G): |dFW| <= G*scale
// parameter offsets: W1 [NH][NIN], b1 [NH], W2 [NH][NH], b2 [NH], W3 [NOUT][NH], b3 [NOUT]
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH;
constexpr int OW3 = OB2 + NH, OB3 = OW3 + NOUT * NH, NPAR = OB3 + NOUT;
static_assert(NPAR == CGFD_MLP_PARAMS, "parameter count of the ABI");

__device__ __forceinline__ float silu(float a) { return a / (1.f + expf(-a)); }
// d silu / da
__device__ __forceinline__ float dsilu(float a) {
  const float s = 1.f / (1.f + expf(-a));
  return s * (1.f + a * (1.f - s));
}

// the parameters as FP32 in shared memory
__device__ void load_params(const __half *w, float *sw) {
  for (int q = threadIdx.x; q < NPAR; q += blockDim.x) sw[q] = __half2float(w[q]);
  __syncthreads();
}

// forward pass of one sample; a1, a2: pre-activations (kept for training)
__device__ void forward(const float *sw, const float *x, float *a1, float *a2, float *y) {
  for (int o = 0; o < NH; ++o) {
    float s = sw[OB1 + o];
    for (int q = 0; q < NIN; ++q) s += sw[OW1 + o * NIN + q] * x[q];
    a1[o] = s;
  }
  for (int o = 0; o < NH; ++o) {
    float s = sw[OB2 + o];
    for (int q = 0; q < NH; ++q) s += sw[OW2 + o * NH + q] * silu(a1[q]);
    a2[o] = s;
  }
  for (int o = 0; o < NOUT; ++o) {
    float s = sw[OB3 + o];
    for (int q = 0; q < NH; ++q) s += sw[OW3 + o * NH + q] * silu(a2[q]);
    y[o] = s;
  }
}

// features of layer cell n: cells[n] = {internal index, normal offset
// (elements), depth in the layer (0: next to the domain's edge), unused}
__device__ bool features(const float *fw, size_t fs, const float *lam2mu, const float *irho,
                         int4 cell, float *x, float *scale, float *zp) {
  const float z = sqrtf(lam2mu[cell.x] / irho[cell.x]);  // rho vp
  float m = 0.f;
  for (int s = 0; s < 5; ++s)
    for (int c = 0; c < 9; ++c) {
      float v = fw[(size_t)c * fs + cell.x + (long)s * cell.y];
      if (c >= 3) v /= z;
      x[s * 9 + c] = v;
      m = fmaxf(m, fabsf(v));
    }
  *zp = z;
  *scale = m;
  // no correction where the field is negligible (and 1/m would overflow)
  if (!(m > MIN_SCALE)) return false;
  const float r = 1.f / m;
  for (int q = 0; q < NIN; ++q) x[q] *= r;
  return true;
}

// corrections of all layer cells into delta [9][n]
__global__ void __launch_bounds__(128) delta_kernel(const float *__restrict__ fw, size_t fs,
                                                    const float *lam2mu, const float *irho,
                                                    const int4 *__restrict__ cells, int n,
                                                    const __half *__restrict__ w,
                                                    const float *__restrict__ gain,
                                                    float *__restrict__ delta) {
  extern __shared__ float sw[];
  load_params(w, sw);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    float x[NIN], a1[NH], a2[NH], y[NOUT], scale, z;
    const int4 cell = cells[q];
    const bool on = features(fw, fs, lam2mu, irho, cell, x, &scale, &z);
    if (on) forward(sw, x, a1, a2, y);
    const float *g = gain + cell.z * NOUT;
    for (int c = 0; c < NOUT; ++c) {
      float d = 0.f;
      if (on) {  // x[0..8]: the cell's own normalised values
        d = g[c] * GAIN * tanhf(y[c] / GAIN);
        d = fminf(fmaxf(d, fminf(0.f, -x[c])), fmaxf(0.f, -x[c]));
      }
      delta[(size_t)c * n + q] = d * scale * (c < 3 ? 1.f : z);
    }
  }
}

__global__ void apply_kernel(float *__restrict__ fw, size_t fs, const int4 *__restrict__ cells,
                             int n, const float *__restrict__ delta) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    for (int c = 0; c < NOUT; ++c) fw[(size_t)c * fs + cells[q].x] += delta[(size_t)c * n + q];
}

// normalised features and scales of all layer cells (training samples)
__global__ void features_kernel(const float *__restrict__ fw, size_t fs, const float *lam2mu,
                                const float *irho, const int4 *__restrict__ cells, int n,
                                float *__restrict__ xs, float *__restrict__ scales,
                                float *__restrict__ zs) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    float x[NIN], scale, z;
    if (!features(fw, fs, lam2mu, irho, cells[q], x, &scale, &z))
      for (int k = 0; k < NIN; ++k) x[k] = 0.f;
    for (int k = 0; k < NIN; ++k) xs[(size_t)q * NIN + k] = x[k];
    scales[q] = scale;
    zs[q] = z;
  }
}

// loss = mean over samples of sum_c (y_c - t_c)^2 and its gradient: one
// thread per sample (grid-stride), gradients summed in shared memory per
// block and then into grad (which the caller zeroes)
constexpr int GRAD_THREADS = 32;
__global__ void __launch_bounds__(GRAD_THREADS)
    grad_kernel(const __half *__restrict__ w, const float *__restrict__ xs,
                const float *__restrict__ ts, int n, float *__restrict__ grad,
                float *__restrict__ loss) {
  extern __shared__ float smem[];
  float *sw = smem;            // NPAR parameters
  float *sg = smem + NPAR;     // NPAR gradient sums
  float *act = sg + NPAR;      // per thread: a1, a2 (2 * NH)
  for (int q = threadIdx.x; q < NPAR; q += blockDim.x) sg[q] = 0.f;
  load_params(w, sw);
  float *a1 = act + threadIdx.x * 2 * NH, *a2 = a1 + NH;
  float lsum = 0.f;
  const float inv_n = 1.f / (float)n;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float x[NIN], y[NOUT], dy[NOUT], d2[NH];
    for (int k = 0; k < NIN; ++k) x[k] = xs[(size_t)s * NIN + k];
    forward(sw, x, a1, a2, y);
    for (int c = 0; c < NOUT; ++c) {
      const float e = y[c] - ts[(size_t)s * NOUT + c];
      lsum += e * e;
      dy[c] = 2.f * e * inv_n;
      atomicAdd(&sg[OB3 + c], dy[c]);
      for (int q = 0; q < NH; ++q) atomicAdd(&sg[OW3 + c * NH + q], dy[c] * silu(a2[q]));
    }
    for (int q = 0; q < NH; ++q) {  // dL/da2
      float s2 = 0.f;
      for (int c = 0; c < NOUT; ++c) s2 += sw[OW3 + c * NH + q] * dy[c];
      d2[q] = s2 * dsilu(a2[q]);
      atomicAdd(&sg[OB2 + q], d2[q]);
    }
    for (int o = 0; o < NH; ++o)
      for (int q = 0; q < NH; ++q) atomicAdd(&sg[OW2 + o * NH + q], d2[o] * silu(a1[q]));
    for (int q = 0; q < NH; ++q) {  // dL/da1, reusing a1's slot
      float s1 = 0.f;
      for (int o = 0; o < NH; ++o) s1 += sw[OW2 + o * NH + q] * d2[o];
      a1[q] = s1 * dsilu(a1[q]);
    }
    for (int o = 0; o < NH; ++o) {
      atomicAdd(&sg[OB1 + o], a1[o]);
      for (int k = 0; k < NIN; ++k) atomicAdd(&sg[OW1 + o * NIN + k], a1[o] * x[k]);
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NPAR; q += blockDim.x) atomicAdd(&grad[q], sg[q]);
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if (threadIdx.x == 0) atomicAdd(loss, lsum * inv_n);
}

}  // namespace mlp

size_t mlp_delta_smem() { return mlp::NPAR * sizeof(float); }

void launch_mlp_step(const float *fw, size_t fs, const float *lam2mu, const float *irho,
                     const int4 *cells, int n, const void *w, const float *gain, float *delta,
                     void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = (n + 127) / 128 < 592 ? (n + 127) / 128 : 592;
  mlp::delta_kernel<<<blocks, 128, mlp_delta_smem(), s>>>(fw, fs, lam2mu, irho, cells, n,
                                                          (const __half *)w, gain, delta);
  mlp::apply_kernel<<<blocks, 128, 0, s>>>(const_cast<float *>(fw), fs, cells, n, delta);
}

void launch_mlp_features(const float *fw, size_t fs, const float *lam2mu, const float *irho,
                         const int4 *cells, int n, float *xs, float *scales, float *zs,
                         void *stream) {
  const int blocks = (n + 127) / 128 < 592 ? (n + 127) / 128 : 592;
  mlp::features_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>(fw, fs, lam2mu, irho, cells, n,
                                                                  xs, scales, zs);
}

}  // namespace cgfd

using namespace cgfd;

extern "C" int cgfd_mlp_gradient(const void *weights_fp16, const float *x, const float *t, int n,
                                 float *grad, float *loss) {
  if (!weights_fp16 || !x || !t || n < 1 || !grad || !loss) {
    set_global_error("cgfd_mlp_gradient: bad arguments");
    return CGFD_ERR_ARG;
  }
  using namespace cgfd::mlp;
  void *dw = nullptr;
  float *dx = nullptr, *dt = nullptr, *dg = nullptr;
  cudaError_t e = cudaMalloc(&dw, NPAR * sizeof(__half));
  if (e == cudaSuccess) e = cudaMalloc(&dx, (size_t)n * NIN * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dt, (size_t)n * NOUT * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dg, (NPAR + 1) * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(dw, weights_fp16, NPAR * sizeof(__half), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, (size_t)n * NIN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dt, t, (size_t)n * NOUT * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dg, 0, (NPAR + 1) * sizeof(float));
  const size_t smem = (2 * NPAR + GRAD_THREADS * 2 * NH) * sizeof(float);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    int blocks = (n + GRAD_THREADS - 1) / GRAD_THREADS;
    if (blocks > 296) blocks = 296;
    grad_kernel<<<blocks, GRAD_THREADS, smem>>>((const __half *)dw, dx, dt, n, dg, dg + NPAR);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(grad, dg, NPAR * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(loss, dg + NPAR, sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dw);
  cudaFree(dx);
  cudaFree(dt);
  cudaFree(dg);
  if (e != cudaSuccess) {
    set_global_error(cudaGetErrorString(e));
    return CGFD_ERR_CUDA;
  }
  return CGFD_OK;
}
