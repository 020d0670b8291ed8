// cgfd_oracle.cpp -- CPU oracle for the CGFD time-stepping path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness checker and the
// timed CPU baseline; the product (copara-cgfd3d_b200/) never links, loads or
// calls it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
//
// It restates, in plain C++ with OpenMP and (by default) FP64 arithmetic, the
// reference's default build (Makefile:8-31: HYindex CFSPML CondFree
// CondFreeVLOW CondFreeTIMG withABS SimpleCar) of the single-GPU hot path:
//   - DRPFD / M22FD / M24FD operators            src/typenew.h:49-87
//   - CalDiffmix (derivatives, VLOW surface)       src/calculate.cu:4121-4275
//   - CalWavemix (RHS, CFS-PML ADE)                src/calculate.cu:4277-4621
//   - CalTIMGmix (traction image, top 3 layers)    src/calculate.cu:5668-5897
//   - LoadForce / LoadMoment                       src/calculate.cu:6130-6255
//   - InterpFocus / ExtractValue + LoadRmom        src/calculate.cu:2586-2643,
//     (focal points)                               1421-1428, 6257-6319
//   - the SrcSmooth spreading of the three kinds    src/calculate.cu:6147-6175,
//     (weights given, 7^3 nodes per source)         6210-6232, 6275-6296
//   - IterationBegin/Inner/Final (RK4 + ADE aux)   src/calculate.cu:6330-6734
//   - RKite stage constants, Tindex                src/calculate.cu:12-13,1355-1422
//   - per-step F/B direction schedule              src/simulation.cc:252-700
//   - PWpick receiver recording                    src/calculate.cu:2780-2830
//   - VelPDcoeff + matinv/matmul                   src/calculate.cu:3320-3466
// and the host pre-processing the kernels consume:
//   - gridmesh::calmetric + mirror_extend          src/gridmesh.cpp:1476-1627,
//                                                  src/common.cpp:97-135
//   - absorb::CalCFSfactors                        src/absorb.cpp:346-805
//   - STF wavelets, cal_stf_moment                 src/mathfunc.cpp:481-608,
//                                                  src/source.cpp:102-131
//   - angle2moment                                 src/source.cpp:134-155
// Parity pin: the reference's own calculate.cu, built single-process from its
// sources by oracle/ref/Makefile, run on the same inputs (tests/golden/).
//
// Layout is the reference's: full arrays (ni+6)(nj+6)(nk+6), g=(i*ny+j)*nz+k.
// The wavefield state is kept like the reference keeps it (FW, W, hW, tW and
// FA/A/hA/tA for the ADE auxiliaries); the stage input copy mW of the
// reference (wavesyn, src/calculate.cu:2956-2991) is not needed because hW is
// complete before W is overwritten.

#include "../include/cgfd.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

enum { VX = 0, VY, VZ, TXX, TYY, TZZ, TXY, TXZ, TYZ };
constexpr int LFD = 3;  // LenFD

// DRP/opt MacCormack one-sided coefficients (src/typenew.h:52-56).
constexpr double DA_1 = -0.30874, DA0 = -0.6326, DA1 = 1.23300, DA2 = -0.3334,
                 DA3 = 0.04168;
// Gottlieb 2-4 MacCormack (src/typenew.h:69-71).
constexpr double MA0 = -1.1666666666666667, MA1 = 1.3333333333333333,
                 MA2 = -0.16666666666666666;
// RK4 coefficients (src/calculate.cu:12-13).
constexpr double RKA[3] = {0.5, 0.5, 1.0};
constexpr double RKB[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

// Direction triples per step%4 and stage (src/simulation.cc:264-641).
constexpr int DIRS[4][4][3] = {
    {{1, 1, 1}, {-1, -1, -1}, {1, 1, 1}, {-1, -1, -1}},
    {{1, 1, -1}, {-1, -1, 1}, {1, 1, -1}, {-1, -1, 1}},
    {{-1, -1, -1}, {1, 1, 1}, {-1, -1, -1}, {1, 1, 1}},
    {{-1, -1, 1}, {1, 1, -1}, {-1, -1, 1}, {1, 1, -1}}};

std::string g_err;

// One-sided DRP derivative: dir>0 reads g-s..g+3s, dir<0 reads g+s..g-3s.
// The sums run in double like the reference (double literals promote the
// expression, src/typenew.h:58-60).
template <class R>
inline double drp(const R *v, long g, long s, int dir, double h) {
  if (dir > 0)
    return (DA_1 * v[g - s] + DA0 * v[g] + DA1 * v[g + s] + DA2 * v[g + 2 * s] +
            DA3 * v[g + 3 * s]) / h;
  return (DA3 * v[g - 3 * s] + DA2 * v[g - 2 * s] + DA1 * v[g - s] + DA0 * v[g] +
          DA_1 * v[g + s]) / (-h);
}
template <class R>
inline double m22(const R *v, long g, long s, int dir, double h) {
  if (dir > 0) return ((double)v[g + s] - v[g]) / h;
  return -1.0 * ((double)v[g] - v[g - s]) / (-h);
}
template <class R>
inline double m24(const R *v, long g, long s, int dir, double h) {
  if (dir > 0) return (MA0 * v[g] + MA1 * v[g + s] + MA2 * v[g + 2 * s]) / h;
  return (MA2 * v[g - 2 * s] + MA1 * v[g - s] + MA0 * v[g]) / (-h);
}
// strF on a 7-point vector centred at index 3 (src/typenew.h:58).
inline double strF7(const double *v, int dir, double h) {
  const int c = 3;
  return (DA_1 * v[c - dir] + DA0 * v[c] + DA1 * v[c + dir] + DA2 * v[c + 2 * dir] +
          DA3 * v[c + 3 * dir]) / (dir * h);
}

template <class R>
struct Solver {
  cgfd_desc d{};
  int nx = 0, ny = 0, nz = 0, top = 0;
  long N = 0;
  std::vector<R> FW[9], W[9], hW[9], tW[9];
  std::vector<R> alpha, beta, rho, zx, zy, zz, jac;
  std::vector<R> APD[3], B[3], DB[3];
  int nab[3] = {0, 0, 0};
  long asz[3] = {0, 0, 0};
  std::vector<R> FA[3][9], A[3][9], hA[3][9], tA[3][9];
  std::vector<double> matVx, matVy;  // nx*ny*9, as matVx2Vz / matVy2Vz
  int nmnt = 0, nfrc = 0, nstfm = 0, nstff = 0;
  std::vector<int> mloc, floc;
  std::vector<double> m6, f3, mstf, fstf;
  int nfoc = 0, fnt = 0;
  double fdt = 0;
  std::vector<int> focloc;
  std::vector<double> smw[3];  // smoothing weights [n][7][7][7]: moments, forces, focal
  std::vector<double> focmom;  // [6][nfoc][fnt]
  int nrecv = 0;
  std::vector<int> rloc;
  std::vector<double> seis;
  int steps = 0;
  bool have_metric = false, have_media = false, have_pml = false, prepared = false;
  // emulated reduced-precision storage of the field sets (orc_set_storage_emulation)
  struct Emul {
    int ebits = 0, mbits = 0;  // 0: off
    int mask = 0;              // 1: W, 2: tW, 4: FW
    int flags = 0;             // 1: tW kept as tW - FW, 2: W kept as W - FW,
                               // 4: FW's rounding residual carried in the tW set,
                               // 8: stochastic rounding
    int adapt = -1;            // >= 0: scales re-chosen every step, max at 2^adapt
    double scale[9] = {1, 1, 1, 1, 1, 1, 1, 1, 1};
  } em;

  long gi(int i, int j, int k) const { return ((long)i * ny + j) * nz + k; }
};

// Round x to a binary format of ebits exponent bits and mbits mantissa bits
// (IEEE layout: bias 2^(ebits-1)-1, subnormals, round to nearest even,
// saturating), e.g. (5, 10) is FP16 and (8, 7) BF16.
double quant_fmt(double x, int ebits, int mbits) {
  if (x == 0.0 || ebits <= 0) return x;
  const int emax = (1 << (ebits - 1)) - 1, emin = 1 - emax;
  int e;
  std::frexp(x, &e);
  const int ex = (e - 1 < emin) ? emin : e - 1;
  const double ulp = std::ldexp(1.0, ex - mbits);
  double q = std::nearbyint(x / ulp) * ulp;
  const double mx = std::ldexp(2.0 - std::ldexp(1.0, -mbits), emax);
  if (q > mx) q = mx;
  if (q < -mx) q = -mx;
  return q;
}

// The same format, rounded stochastically: up with probability equal to the
// fraction of an ulp above the lower neighbour (u uniform in [0, 1)).
double quant_fmt_sr(double x, int ebits, int mbits, double u) {
  if (x == 0.0 || ebits <= 0) return x;
  const int emax = (1 << (ebits - 1)) - 1, emin = 1 - emax;
  int e;
  std::frexp(x, &e);
  const int ex = (e - 1 < emin) ? emin : e - 1;
  const double ulp = std::ldexp(1.0, ex - mbits);
  double q = std::floor(x / ulp + u) * ulp;
  const double mx = std::ldexp(2.0 - std::ldexp(1.0, -mbits), emax);
  if (q > mx) q = mx;
  if (q < -mx) q = -mx;
  return q;
}

// uniform [0, 1) from a 64-bit key (splitmix64 finaliser)
double hash_unit(uint64_t k) {
  k += 0x9E3779B97F4A7C15ull;
  k = (k ^ (k >> 30)) * 0xBF58476D1CE4E5B9ull;
  k = (k ^ (k >> 27)) * 0x94D049BB133111EBull;
  k ^= k >> 31;
  return (double)(k >> 11) * 0x1.0p-53;
}

struct Handle {
  int prec;  // 0 = double, 1 = float
  void *s;
  std::string err;
};

template <class R>
int init(Solver<R> &S, const cgfd_desc &d, std::string &err) {
  if (d.ni < 1 || d.nj < 1 || d.nk < 4 || d.steph <= 0 || d.stept <= 0 || d.nt < 0) {
    err = "bad grid or step sizes";
    return CGFD_ERR_ARG;
  }
  if (d.hybrid_grid != 1) {
    err = "only hybrid_grid=1 is supported (SimpleCar build)";
    return CGFD_ERR_ARG;
  }
  for (int q = 0; q < 6; ++q)
    if (d.nabs[q] < 0) { err = "negative nabs"; return CGFD_ERR_ARG; }
  if (d.nabs[5] != 0) { err = "nabs[5] (top) must be 0: free surface"; return CGFD_ERR_ARG; }
  if (d.nabs[0] + d.nabs[1] > d.ni || d.nabs[2] + d.nabs[3] > d.nj ||
      d.nabs[4] + d.nabs[5] > d.nk) {
    err = "PML wider than the grid";
    return CGFD_ERR_ARG;
  }
  if (d.con_index < LFD || d.con_index > d.nk + LFD - 1) {
    err = "con_index must lie in [3, nk+2]";
    return CGFD_ERR_ARG;
  }
  S.d = d;
  S.nx = d.ni + 2 * LFD; S.ny = d.nj + 2 * LFD; S.nz = d.nk + 2 * LFD;
  S.top = d.nk + LFD - 1;
  S.N = (long)S.nx * S.ny * S.nz;
  for (int c = 0; c < 9; ++c) {
    S.FW[c].assign(S.N, 0); S.W[c].assign(S.N, 0);
    S.hW[c].assign(S.N, 0); S.tW[c].assign(S.N, 0);
  }
  S.nab[0] = d.nabs[0] + d.nabs[1];
  S.nab[1] = d.nabs[2] + d.nabs[3];
  S.nab[2] = d.nabs[4] + d.nabs[5];
  S.asz[0] = (long)S.nab[0] * S.ny * S.nz;
  S.asz[1] = (long)S.nab[1] * S.nx * S.nz;
  S.asz[2] = (long)S.nab[2] * S.nx * S.ny;
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 9; ++c) {
      S.FA[a][c].assign(S.asz[a], 0); S.A[a][c].assign(S.asz[a], 0);
      S.hA[a][c].assign(S.asz[a], 0); S.tA[a][c].assign(S.asz[a], 0);
    }
  S.seis.assign((size_t)9 * 0, 0);
  return CGFD_OK;
}

// 3x3 Gauss-Jordan inverse without pivoting, row-major, the reference's loop
// order (src/calculate.cu:3444-3466).
void matinv3(double *a) {
  const int n = 3;
  for (int i = 0; i < n; ++i) {
    double con = a[i * n + i];
    a[i * n + i] = 1;
    for (int j = 0; j < n; ++j) a[i * n + j] /= con;
    for (int j = 0; j < n; ++j)
      if (j != i) {
        con = a[j * n + i];
        a[j * n + i] = 0;
        for (int k = 0; k < n; ++k) a[j * n + k] -= a[i * n + k] * con;
      }
  }
}
void matmul3(const double *a, const double *b, double *c) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += a[i * 3 + k] * b[k * 3 + j];
      c[i * 3 + j] = s;
    }
}

// VelPDcoeff (src/calculate.cu:3320-3428) under SimpleCar: xi = (1,0,0),
// eta = (0,1,0); zeta from the metric at the surface layer.
template <class R>
void vel_pd_coeff(Solver<R> &S) {
  S.matVx.assign((size_t)S.nx * S.ny * 9, 0.0);
  S.matVy.assign((size_t)S.nx * S.ny * 9, 0.0);
  const int k = S.top;
  for (int i = LFD; i < S.d.ni + LFD; ++i)
    for (int j = LFD; j < S.d.nj + LFD; ++j) {
      const long g = S.gi(i, j, k);
      const double Bzx = (double)S.B[2][k] / S.B[0][i];
      const double Bzy = (double)S.B[2][k] / S.B[1][j];
      const double miu = (double)S.rho[g] * S.beta[g] * S.beta[g];
      const double lam2mu = (double)S.rho[g] * S.alpha[g] * S.alpha[g];
      const double lam = lam2mu - 2.0 * miu;
      const double e11 = 1, e12 = 0, e13 = 0, e21 = 0, e22 = 1, e23 = 0;
      const double e31 = S.zx[g], e32 = S.zy[g], e33 = S.zz[g];
      double Am[9], Bm[9], Cm[9], t[9];
      Am[0] = lam2mu * e31 * e31 + miu * (e32 * e32 + e33 * e33);
      Am[1] = lam * e31 * e32 + miu * e32 * e31;
      Am[2] = lam * e31 * e33 + miu * e33 * e31;
      Am[3] = lam * e32 * e31 + miu * e31 * e32;
      Am[4] = lam2mu * e32 * e32 + miu * (e31 * e31 + e33 * e33);
      Am[5] = lam * e32 * e33 + miu * e33 * e32;
      Am[6] = lam * e33 * e31 + miu * e31 * e33;
      Am[7] = lam * e33 * e32 + miu * e32 * e33;
      Am[8] = lam2mu * e33 * e33 + miu * (e31 * e31 + e32 * e32);
      matinv3(Am);
      Bm[0] = lam2mu * e31 * e11 + miu * (e32 * e12 + e33 * e13);
      Bm[1] = lam * e31 * e12 + miu * e32 * e11;
      Bm[2] = lam * e31 * e13 + miu * e33 * e11;
      Bm[3] = lam * e32 * e11 + miu * e31 * e12;
      Bm[4] = lam2mu * e32 * e12 + miu * (e31 * e11 + e33 * e13);
      Bm[5] = lam * e32 * e13 + miu * e33 * e12;
      Bm[6] = lam * e33 * e11 + miu * e31 * e13;
      Bm[7] = lam * e33 * e12 + miu * e32 * e13;
      Bm[8] = lam2mu * e33 * e13 + miu * (e32 * e12 + e31 * e11);
      Cm[0] = lam2mu * e31 * e21 + miu * (e32 * e22 + e33 * e23);
      Cm[1] = lam * e31 * e22 + miu * e32 * e21;
      Cm[2] = lam * e31 * e23 + miu * e33 * e21;
      Cm[3] = lam * e32 * e21 + miu * e31 * e22;
      Cm[4] = lam2mu * e32 * e22 + miu * (e31 * e21 + e33 * e23);
      Cm[5] = lam * e32 * e23 + miu * e33 * e22;
      Cm[6] = lam * e33 * e21 + miu * e31 * e23;
      Cm[7] = lam * e33 * e22 + miu * e32 * e23;
      Cm[8] = lam2mu * e33 * e23 + miu * (e31 * e21 + e32 * e22);
      const size_t m = ((size_t)i * S.ny + j) * 9;
      matmul3(Am, Bm, t);
      for (int q = 0; q < 9; ++q) S.matVx[m + q] = -1 * t[q] * Bzx;
      matmul3(Am, Cm, t);
      for (int q = 0; q < 9; ++q) S.matVy[m + q] = -1 * t[q] * Bzy;
    }
}

// Derivatives + RHS + CFS-PML of one stage: CalDiffmix (4121-4275) then
// CalWavemix (4277-4621).  Writes hW and hA.
template <class R>
void rhs(Solver<R> &S, int rk, int X, int Y, int Z) {
  auto &in = (rk == 0) ? S.FW : S.W;
  auto &ain = (rk == 0) ? S.FA : S.A;
  const int ni = S.d.ni, nj = S.d.nj, nk = S.d.nk;
  const int *nabs = S.d.nabs;
  const long sx = (long)S.ny * S.nz, sy = S.nz, sz = 1;
  const double h = S.d.steph;
  const int top = S.top, con = S.d.con_index;
  const R *Vx = in[VX].data(), *Vy = in[VY].data(), *Vz = in[VZ].data();
  const R *Txx = in[TXX].data(), *Tyy = in[TYY].data(), *Tzz = in[TZZ].data();
  const R *Txy = in[TXY].data(), *Txz = in[TXZ].data(), *Tyz = in[TYZ].data();
#pragma omp parallel for schedule(static)
  for (int i = LFD; i < ni + LFD; ++i)
    for (int j = LFD; j < nj + LFD; ++j)
      for (int k = LFD; k < nk + LFD; ++k) {
        const long g = S.gi(i, j, k);
        // ---- CalDiffmix: directional derivatives (stored as R like pd) ----
        const R DxTxx = drp(Txx, g, sx, X, h), DxTxy = drp(Txy, g, sx, X, h),
                DxTxz = drp(Txz, g, sx, X, h), DxVx = drp(Vx, g, sx, X, h),
                DxVy = drp(Vy, g, sx, X, h), DxVz = drp(Vz, g, sx, X, h);
        const R DyTyy = drp(Tyy, g, sy, Y, h), DyTxy = drp(Txy, g, sy, Y, h),
                DyTyz = drp(Tyz, g, sy, Y, h), DyVx = drp(Vx, g, sy, Y, h),
                DyVy = drp(Vy, g, sy, Y, h), DyVz = drp(Vz, g, sy, Y, h);
        const R DzTzz = drp(Tzz, g, sz, Z, h), DzTxz = drp(Txz, g, sz, Z, h),
                DzTyz = drp(Tyz, g, sz, Z, h);
        const bool curved = k >= con;
        R DzTxx = 0, DzTyy = 0, DzTxy = 0;
        if (curved) {
          DzTxx = drp(Txx, g, sz, Z, h);
          DzTyy = drp(Tyy, g, sz, Z, h);
          DzTxy = drp(Txy, g, sz, Z, h);
        }
        const size_t m = ((size_t)i * S.ny + j) * 9;
        R DzVx, DzVy, DzVz;
        if (k == top) {
          const double *cx = &S.matVx[m], *cy = &S.matVy[m];
          DzVx = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz + cy[0] * DyVx +
                 cy[1] * DyVy + cy[2] * DyVz;
          DzVy = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz + cy[3] * DyVx +
                 cy[4] * DyVy + cy[5] * DyVz;
          DzVz = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz + cy[6] * DyVx +
                 cy[7] * DyVy + cy[8] * DyVz;
        } else if (k == top - 1) {
          DzVx = m22(Vx, g, sz, Z, h); DzVy = m22(Vy, g, sz, Z, h); DzVz = m22(Vz, g, sz, Z, h);
        } else if (k == top - 2) {
          DzVx = m24(Vx, g, sz, Z, h); DzVy = m24(Vy, g, sz, Z, h); DzVz = m24(Vz, g, sz, Z, h);
        } else {
          DzVx = drp(Vx, g, sz, Z, h); DzVy = drp(Vy, g, sz, Z, h); DzVz = drp(Vz, g, sz, Z, h);
        }
        // ---- CalWavemix: RHS ----
        R rho = S.rho[g];
        const R miu = rho * S.beta[g] * S.beta[g];
        const R lam2mu = rho * S.alpha[g] * S.alpha[g];
        const R lambda = lam2mu - 2.0 * miu;
        rho = 1.0 / rho;
        const R ztz = S.zz[g];
        // Below ConIndex the reference uses zeta_z only (4409-4458); with
        // ztx=zty=0 and the unused z-derivatives at 0 the curved formulas
        // reduce to exactly those expressions.
        const R ztx = curved ? S.zx[g] : R(0), zty = curved ? S.zy[g] : R(0);
        const R DxiVx = DxTxx * rho, DetVx = DyTxy * rho,
                DztVx = (ztx * DzTxx + zty * DzTxy + ztz * DzTxz) * rho;
        const R DxiVy = DxTxy * rho, DetVy = DyTyy * rho,
                DztVy = (ztx * DzTxy + zty * DzTyy + ztz * DzTyz) * rho;
        const R DxiVz = DxTxz * rho, DetVz = DyTyz * rho,
                DztVz = (ztx * DzTxz + zty * DzTyz + ztz * DzTzz) * rho;
        const R DxiTxx = lam2mu * DxVx, DetTxx = lambda * DyVy,
                DztTxx = lam2mu * ztx * DzVx + lambda * zty * DzVy + lambda * ztz * DzVz;
        const R DxiTyy = lambda * DxVx, DetTyy = lam2mu * DyVy,
                DztTyy = lambda * ztx * DzVx + lam2mu * zty * DzVy + lambda * ztz * DzVz;
        const R DxiTzz = lambda * DxVx, DetTzz = lambda * DyVy,
                DztTzz = lambda * ztx * DzVx + lambda * zty * DzVy + lam2mu * ztz * DzVz;
        const R DxiTxy = DxVy * miu, DetTxy = DyVx * miu,
                DztTxy = (zty * DzVx + ztx * DzVy) * miu;
        const R DxiTxz = DxVz * miu, DetTxz = 0,
                DztTxz = (ztz * DzVx + ztx * DzVz) * miu;
        const R DxiTyz = 0, DetTyz = DyVz * miu,
                DztTyz = (ztz * DzVy + zty * DzVz) * miu;
        const R Bx = S.B[0][i], By = S.B[1][j], Bz = S.B[2][k];
        const R APDx = S.APD[0][i], APDy = S.APD[1][j], APDz = S.APD[2][k];
        const R DBx = S.DB[0][i], DBy = S.DB[1][j], DBz = S.DB[2][k];
        const R dxi[9] = {DxiVx, DxiVy, DxiVz, DxiTxx, DxiTyy, DxiTzz, DxiTxy, DxiTxz, DxiTyz};
        const R det[9] = {DetVx, DetVy, DetVz, DetTxx, DetTyy, DetTzz, DetTxy, DetTxz, DetTyz};
        const R dzt[9] = {DztVx, DztVy, DztVz, DztTxx, DztTyy, DztTzz, DztTxy, DztTxz, DztTyz};
        R hw[9];
        for (int c = 0; c < 9; ++c) hw[c] = dxi[c] / Bx + det[c] / By + dzt[c] / Bz;
        // top-surface split of dV/dzeta into its xi and eta parts (4479-4491)
        R DzVx1 = 0, DzVx2 = 0, DzVy1 = 0, DzVy2 = 0, DzVz1 = 0, DzVz2 = 0;
        if (k == top) {
          const double *cx = &S.matVx[m], *cy = &S.matVy[m];
          DzVx1 = cx[0] * DxVx + cx[1] * DxVy + cx[2] * DxVz;
          DzVx2 = cy[0] * DyVx + cy[1] * DyVy + cy[2] * DyVz;
          DzVy1 = cx[3] * DxVx + cx[4] * DxVy + cx[5] * DxVz;
          DzVy2 = cy[3] * DyVx + cy[4] * DyVy + cy[5] * DyVz;
          DzVz1 = cx[6] * DxVx + cx[7] * DxVy + cx[8] * DxVz;
          DzVz2 = cy[6] * DyVx + cy[7] * DyVy + cy[8] * DyVz;
        }
        if (i <= nabs[0] + LFD - 1 || i >= ni + LFD - nabs[1]) {
          const int xa = (i < nabs[0] + LFD) ? i - LFD : i - (ni + LFD - nabs[1]) + nabs[0];
          const long p = ((long)xa * S.ny + j) * S.nz + k;
          for (int c = 0; c < 9; ++c) hw[c] -= ain[0][c][p] / Bx;
          for (int c = 0; c < 9; ++c) S.hA[0][c][p] = dxi[c] * DBx - APDx * ain[0][c][p];
          if (k == top) {
            S.hA[0][TXX][p] += DBx * Bx * (lam2mu * ztx * DzVx1 + lambda * zty * DzVy1 + lambda * ztz * DzVz1);
            S.hA[0][TYY][p] += DBx * Bx * (lambda * ztx * DzVx1 + lam2mu * zty * DzVy1 + lambda * ztz * DzVz1);
            S.hA[0][TZZ][p] += DBx * Bx * (lambda * ztx * DzVx1 + lambda * zty * DzVy1 + lam2mu * ztz * DzVz1);
            S.hA[0][TXY][p] += DBx * Bx * (zty * DzVx1 + ztx * DzVy1) * miu;
            S.hA[0][TXZ][p] += DBx * Bx * (ztz * DzVx1 + ztx * DzVz1) * miu;
            S.hA[0][TYZ][p] += DBx * Bx * (ztz * DzVy1 + zty * DzVz1) * miu;
          }
        }
        if (j <= nabs[2] + LFD - 1 || j >= nj + LFD - nabs[3]) {
          const int ya = (j < nabs[2] + LFD) ? j - LFD : j - (nj + LFD - nabs[3]) + nabs[2];
          const long p = ((long)ya * S.nx + i) * S.nz + k;
          for (int c = 0; c < 9; ++c) hw[c] -= ain[1][c][p] / By;
          for (int c = 0; c < 9; ++c) S.hA[1][c][p] = det[c] * DBy - APDy * ain[1][c][p];
          if (k == top) {
            S.hA[1][TXX][p] += DBy * By * (lam2mu * ztx * DzVx2 + lambda * zty * DzVy2 + lambda * ztz * DzVz2);
            S.hA[1][TYY][p] += DBy * By * (lambda * ztx * DzVx2 + lam2mu * zty * DzVy2 + lambda * ztz * DzVz2);
            S.hA[1][TZZ][p] += DBy * By * (lambda * ztx * DzVx2 + lambda * zty * DzVy2 + lam2mu * ztz * DzVz2);
            S.hA[1][TXY][p] += DBy * By * (zty * DzVx2 + ztx * DzVy2) * miu;
            S.hA[1][TXZ][p] += DBy * By * (ztz * DzVx2 + ztx * DzVz2) * miu;
            S.hA[1][TYZ][p] += DBy * By * (ztz * DzVy2 + zty * DzVz2) * miu;
          }
        }
        if (k <= nabs[4] + LFD - 1 || k >= nk + LFD - nabs[5]) {
          const int za = (k < nabs[4] + LFD) ? k - LFD : k - (nk + LFD - nabs[5]) + nabs[4];
          const long p = ((long)za * S.nx + i) * S.ny + j;
          for (int c = 0; c < 9; ++c) hw[c] -= ain[2][c][p] / Bz;
          for (int c = 0; c < 9; ++c) S.hA[2][c][p] = dzt[c] * DBz - APDz * ain[2][c][p];
        }
        for (int c = 0; c < 9; ++c) S.hW[c][g] = hw[c];
      }
}

// CalTIMGmix (src/calculate.cu:5668-5897): velocity RHS of the top 3 layers
// from the conservative momentum equation with the normal traction imaged
// antisymmetrically about the surface (traction-free).
template <class R>
void timg(Solver<R> &S, int rk, int X, int Y, int Z) {
  auto &in = (rk == 0) ? S.FW : S.W;
  auto &ain = (rk == 0) ? S.FA : S.A;
  const int ni = S.d.ni, nj = S.d.nj, nk = S.d.nk;
  const int *nabs = S.d.nabs;
  const long sx = (long)S.ny * S.nz, sy = S.nz;
  const double h = S.d.steph;
  // component c of dV/dt uses stresses (T1,T2,T3) contracted with (xi,eta,zeta)
  const int TC[3][3] = {{TXX, TXY, TXZ}, {TXY, TYY, TYZ}, {TXZ, TYZ, TZZ}};
#pragma omp parallel for schedule(static)
  for (int i = LFD; i < ni + LFD; ++i)
    for (int j = LFD; j < nj + LFD; ++j)
      for (int cz = 0; cz < LFD; ++cz) {
        const int k = nk + cz;
        const long g = S.gi(i, j, k);
        const double rhojac = 1.0 / (double)S.rho[g] / (double)S.jac[g];
        const R Bx = S.B[0][i], By = S.B[1][j];
        const R APDx = S.APD[0][i], APDy = S.APD[1][j];
        const R DBx = S.DB[0][i], DBy = S.DB[1][j];
        const int s = 2 - cz;  // surface lies s layers above this one
        for (int c = 0; c < 3; ++c) {
          const R *T1 = in[TC[c][0]].data(), *T2 = in[TC[c][1]].data(),
                  *T3 = in[TC[c][2]].data();
          double vx[7], vy[7], vz[7];
          for (int n = 0; n < 7; ++n) {
            const long gx = g + (n - 3) * sx, gy = g + (n - 3) * sy, gz = g + (n - 3);
            vx[n] = (R)(S.jac[gx] * T1[gx]);
            vy[n] = (R)(S.jac[gy] * T2[gy]);
            vz[n] = (R)(S.jac[gz] * (S.zx[gz] * T1[gz] + S.zy[gz] * T2[gz] + S.zz[gz] * T3[gz]));
          }
          for (int q = 1; q <= LFD - s; ++q) vz[3 + s + q] = -vz[3 + s - q];
          vz[3 + s] = 0.0;
          const R DxT = rhojac * strF7(vx, X, h);
          const R DyT = rhojac * strF7(vy, Y, h);
          const R DzT = rhojac * strF7(vz, Z, h);
          R hv = DxT / Bx + DyT / By + DzT;
          if (i <= nabs[0] + LFD - 1 || i >= ni + LFD - nabs[1]) {
            const int xa = (i < nabs[0] + LFD) ? i - LFD : i - (ni + LFD - nabs[1]) + nabs[0];
            const long p = ((long)xa * S.ny + j) * S.nz + k;
            hv -= ain[0][c][p] / Bx;
            S.hA[0][c][p] = DBx * DxT - APDx * ain[0][c][p];
          }
          if (j <= nabs[2] + LFD - 1 || j >= nj + LFD - nabs[3]) {
            const int ya = (j < nabs[2] + LFD) ? j - LFD : j - (nj + LFD - nabs[3]) + nabs[2];
            const long p = ((long)ya * S.nx + i) * S.nz + k;
            hv -= ain[1][c][p] / By;
            S.hA[1][c][p] = DBy * DyT - APDy * ain[1][c][p];
          }
          S.hW[c][g] = hv;
        }
      }
}

// ExtractValue (src/calculate.cu:2586-2613): the series at time t, linear
// between samples PL = floor(t/DT) and PL + 1 (PR = PL when t is within 1e-5
// of a sample), zero outside [0, DT*(n-1)].
inline double extract_value(const double *stf, int n, double DT, double time) {
  const double Tend = DT * (n - 1);
  if (time > Tend || time < 0) return 0;
  int PL = (int)(time / DT);
  int PR = (std::fabs(time - DT * std::floor(time / DT)) < 1e-5) ? PL : PL + 1;
  PL = std::min(PL, n - 1);
  PR = std::min(PR, n - 1);
  return stf[PL] + (stf[PR] - stf[PL]) * ((time - DT * PL) / DT);
}

// The node (i+a-3, j+b-3, k+c-3) of a smoothed source at (i, j, k) takes
// the fraction w[a][b][c]; valid nodes only (SrcSmooth branches of the
// three Load kernels).  Unsmoothed: the source's own node, w = 1.
template <class R, class F>
void spread(const Solver<R> &S, const std::vector<double> &w, int q, const int *l, F &&f) {
  if (w.empty()) {
    f(l[0], l[1], l[2], 1.0);
    return;
  }
  for (int a = 0; a < 7; ++a)
    for (int b = 0; b < 7; ++b)
      for (int c = 0; c < 7; ++c) {
        const int i = l[0] + a - 3, j = l[1] + b - 3, k = l[2] + c - 3;
        if (i < LFD || i >= S.d.ni + LFD || j < LFD || j >= S.d.nj + LFD || k < LFD ||
            k >= S.d.nk + LFD)
          continue;
        f(i, j, k, w[(size_t)343 * q + (a * 7 + b) * 7 + c]);
      }
}

// LoadForce / LoadMoment (src/calculate.cu:6130-6255), Tindex = 2*currT+tinc;
// focal points as LoadRmom (6257-6319) at time (currT + tinc/2)*stept.
template <class R>
void sources(Solver<R> &S, int tindex, double time) {
  const double h3 = S.d.steph * S.d.steph * S.d.steph;
  for (int q = 0; q < S.nfoc; ++q) {
    double M[6];
    for (int c = 0; c < 6; ++c)
      M[c] = extract_value(&S.focmom[((size_t)c * S.nfoc + q) * S.fnt], S.fnt, S.fdt, time);
    spread(S, S.smw[2], q, &S.focloc[3 * q], [&](int i, int j, int k, double w) {
      const long g = S.gi(i, j, k);
      const double A = w / (h3 * (double)S.jac[g]);
      for (int c = 0; c < 6; ++c) S.hW[TXX + c][g] -= (R)(M[c] * A);
    });
  }
  for (int q = 0; q < S.nfrc; ++q) {
    const R stf = S.fstf[(size_t)q * S.nstff + tindex];
    spread(S, S.smw[1], q, &S.floc[3 * q], [&](int i, int j, int k, double w) {
      const long g = S.gi(i, j, k);
      R Aa = h3 * S.jac[g];
      Aa = (R)w / (Aa * S.rho[g]);
      if (k == S.top) Aa = Aa * 2.0;
      S.hW[VX][g] += stf * (R)S.f3[3 * q] * Aa;
      S.hW[VY][g] += stf * (R)S.f3[3 * q + 1] * Aa;
      S.hW[VZ][g] += stf * (R)S.f3[3 * q + 2] * Aa;
    });
  }
  for (int q = 0; q < S.nmnt; ++q) {
    const R stf = S.mstf[(size_t)q * S.nstfm + tindex];
    spread(S, S.smw[0], q, &S.mloc[3 * q], [&](int i, int j, int k, double w) {
      const long g = S.gi(i, j, k);
      const R Aa = stf * (R)w / (h3 * S.jac[g]);
      for (int c = 0; c < 6; ++c) S.hW[TXX + c][g] -= (R)S.m6[6 * q + c] * Aa;
    });
  }
}

// IterationBegin / Inner / Final (src/calculate.cu:6330-6734) for the
// wavefield (valid cells) and the ADE auxiliaries.
// The same update with the stored sets rounded as the 16-bit storage of
// the solver keeps them (test infrastructure: localises the storage error).
// The first stage writes no tW; the second rebuilds it from the rounded
// stage output, tW = FW + (b0/a0)(W - FW) + b1 dt H, as the solver does.
template <class R>
void update_emulated(Solver<R> &S, int rk) {
  const auto &E = S.em;
  const double a = (rk < 3) ? RKA[rk] * S.d.stept : 0.0;
  const double b = RKB[rk] * S.d.stept;
  const int ni = S.d.ni, nj = S.d.nj, nk = S.d.nk;
  const bool block = E.ebits >= 100;  // block floating point: rounded below, per block
  const bool fb = (E.flags & 4) != 0;   // requires flags & 1 (checked at set-up)
  const bool sr = (E.flags & 8) != 0;
  const uint64_t stage_key = ((uint64_t)S.steps * 4 + (uint64_t)rk) << 40;
  // v rounded as set `set` stores component c of cell p
  auto qp = [&](double v, int c, int set, long p) {
    if (!(E.mask & set) || block) return v;
    if (sr) {
      const uint64_t key = stage_key ^ ((uint64_t)p * 64 + (uint64_t)c * 8 + (uint64_t)set);
      return quant_fmt_sr(v / E.scale[c], E.ebits, E.mbits, hash_unit(key)) * E.scale[c];
    }
    return quant_fmt(v / E.scale[c], E.ebits, E.mbits) * E.scale[c];
  };
#pragma omp parallel for schedule(static)
  for (int i = LFD; i < ni + LFD; ++i)
    for (int j = LFD; j < nj + LFD; ++j)
      for (int k = LFD; k < nk + LFD; ++k) {
        const long p = S.gi(i, j, k);
        auto q = [&](double v, int c, int set) { return qp(v, c, set, p); };
        for (int c = 0; c < 9; ++c) {
          const double f = S.FW[c][p], h = S.hW[c][p], w = S.W[c][p];
          const double dtw = (E.flags & 1) ? 1.0 : 0.0, dw = (E.flags & 2) ? 1.0 : 0.0;
          if (rk == 0) {
            S.W[c][p] = (R)(dw * f + q(f * (1 - dw) + a * h, c, 1));
          } else if (rk < 3) {
            double t;
            if (rk == 1) {
              t = (RKB[0] / RKA[0]) * (w - f) + b * h + (1 - dtw) * f;
              // error feedback: the tW set still holds FW + r, r the part of
              // the last step's new state that FW's rounding dropped
              if (fb) t += (double)S.tW[c][p] - f;
            } else {
              t = S.tW[c][p] - dtw * f + b * h;
            }
            S.tW[c][p] = (R)(dtw * f + q(t, c, 2));
            S.W[c][p] = (R)(dw * f + q(f * (1 - dw) + a * h, c, 1));
          } else {
            const double ex = S.tW[c][p] + b * h, wn = q(ex, c, 4);
            S.W[c][p] = (R)wn;
            // error feedback: keep the rounding residual as the tW set's
            // difference from the new state (read back in the next step's
            // second stage; the first stage does not touch the tW set)
            if (fb) S.tW[c][p] = (R)(wn + q(ex - wn, c, 2));
          }
        }
      }
  if (!block) return;
  // block floating point: every run of B x-adjacent valid cells shares one
  // exponent, each value keeps a sign and mbits magnitude bits below it
  const int B = E.ebits - 100;
  auto qblock = [&](std::vector<R> *set, std::vector<R> *base, bool delta) {
#pragma omp parallel for schedule(static)
    for (int j = LFD; j < nj + LFD; ++j)
      for (int k = LFD; k < nk + LFD; ++k)
        for (int c = 0; c < 9; ++c)
          for (int i0 = 0; i0 < ni; i0 += B) {
            const int i1 = std::min(i0 + B, ni);
            double mx = 0;
            for (int i = i0; i < i1; ++i) {
              const long p = S.gi(i + LFD, j, k);
              const double v = set[c][p] - (delta ? (double)base[c][p] : 0.0);
              mx = std::max(mx, std::fabs(v));
            }
            if (mx == 0) continue;
            int e;
            std::frexp(mx, &e);  // mx < 2^e
            const double ulp = std::ldexp(1.0, e - E.mbits);
            for (int i = i0; i < i1; ++i) {
              const long p = S.gi(i + LFD, j, k);
              const double bv = delta ? (double)base[c][p] : 0.0;
              const double v = set[c][p] - bv;
              set[c][p] = (R)(bv + std::nearbyint(v / ulp) * ulp);
            }
          }
  };
  if (rk < 3) {
    if (E.mask & 1) qblock(S.W, S.FW, (E.flags & 2) != 0);
    if ((E.mask & 2) && rk > 0) qblock(S.tW, S.FW, (E.flags & 1) != 0);
  } else {
    // the loop left the exact new state in W (and, with error feedback, in tW)
    if (E.mask & 4) qblock(S.W, S.FW, false);
    if (fb && (E.mask & 2)) qblock(S.tW, S.W, true);  // the residual, against the new FW
  }
}

template <class R>
void update(Solver<R> &S, int rk) {
  const R a = (rk < 3) ? (R)(RKA[rk] * S.d.stept) : R(0);
  const R b = (R)(RKB[rk] * S.d.stept);
  const int ni = S.d.ni, nj = S.d.nj, nk = S.d.nk;
  auto upd = [&](std::vector<R> *Fv, std::vector<R> *Wv, std::vector<R> *Hv,
                 std::vector<R> *Tv, long p) {
    for (int c = 0; c < 9; ++c) {
      const R hh = Hv[c][p];
      if (rk == 0) {
        Wv[c][p] = Fv[c][p] + a * hh;
        Tv[c][p] = Fv[c][p] + b * hh;
      } else if (rk < 3) {
        Wv[c][p] = Fv[c][p] + a * hh;
        Tv[c][p] = Tv[c][p] + b * hh;
      } else {
        Wv[c][p] = Tv[c][p] + b * hh;
      }
    }
  };
  if (S.em.ebits > 0) update_emulated(S, rk);
  else {
#pragma omp parallel for schedule(static)
  for (int i = LFD; i < ni + LFD; ++i)
    for (int j = LFD; j < nj + LFD; ++j)
      for (int k = LFD; k < nk + LFD; ++k) upd(S.FW, S.W, S.hW, S.tW, S.gi(i, j, k));
  }
#pragma omp parallel for schedule(static)
  for (int xa = 0; xa < S.nab[0]; ++xa)
    for (int j = LFD; j < nj + LFD; ++j)
      for (int k = LFD; k < nk + LFD; ++k)
        upd(S.FA[0], S.A[0], S.hA[0], S.tA[0], ((long)xa * S.ny + j) * S.nz + k);
#pragma omp parallel for schedule(static)
  for (int ya = 0; ya < S.nab[1]; ++ya)
    for (int i = LFD; i < ni + LFD; ++i)
      for (int k = LFD; k < nk + LFD; ++k)
        upd(S.FA[1], S.A[1], S.hA[1], S.tA[1], ((long)ya * S.nx + i) * S.nz + k);
#pragma omp parallel for schedule(static)
  for (int za = 0; za < S.nab[2]; ++za)
    for (int i = LFD; i < ni + LFD; ++i)
      for (int j = LFD; j < nj + LFD; ++j)
        upd(S.FA[2], S.A[2], S.hA[2], S.tA[2], ((long)za * S.nx + i) * S.ny + j);
}

template <class R>
int rk_stage(Solver<R> &S, int rk, int curr_t, int X, int Y, int Z, std::string &err) {
  if (!(S.have_metric && S.have_media && S.have_pml)) {
    err = "metric, media and PML must be uploaded first";
    return CGFD_ERR_STATE;
  }
  if (rk < 0 || rk > 3 || (X != 1 && X != -1) || (Y != 1 && Y != -1) || (Z != 1 && Z != -1)) {
    err = "bad stage arguments";
    return CGFD_ERR_ARG;
  }
  if (!S.prepared) { vel_pd_coeff(S); S.prepared = true; }
  const int tinc = (rk == 0) ? 0 : (rk < 3 ? 1 : 2);
  const int tindex = 2 * curr_t + tinc;
  if ((S.nmnt && tindex >= S.nstfm) || (S.nfrc && tindex >= S.nstff)) {
    err = "source time function too short for this step";
    return CGFD_ERR_ARG;
  }
  rhs(S, rk, X, Y, Z);
  timg(S, rk, X, Y, Z);
  sources(S, tindex, (curr_t + tinc * 0.5) * S.d.stept);
  update(S, rk);
  if (rk == 3) {  // wavesyn(FW, W); abssyn(3)
    for (int c = 0; c < 9; ++c) S.FW[c] = S.W[c];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 9; ++c) S.FA[a][c] = S.A[a][c];
    if (S.em.ebits > 0 && S.em.adapt >= 0) {  // emulation: scales from this step's maxima
      for (int c = 0; c < 9; ++c) {
        double mx = 0;
        for (long p = 0; p < S.N; ++p) mx = std::max(mx, (double)std::fabs(S.FW[c][p]));
        if (mx > 0) {
          int e;
          std::frexp(mx, &e);
          S.em.scale[c] = std::ldexp(1.0, e - S.em.adapt);
        }
      }
    }
  }
  return CGFD_OK;
}

template <class R>
int step(Solver<R> &S, int n, std::string &err) {
  for (int s = 0; s < n; ++s) {
    const int t = S.steps;
    if (S.nrecv && t >= S.d.nt) { err = "seismogram buffer full (nt steps)"; return CGFD_ERR_ARG; }
    for (int rk = 0; rk < 4; ++rk) {
      const int *dd = DIRS[t % 4][rk];
      const int st = rk_stage(S, rk, t, dd[0], dd[1], dd[2], err);
      if (st) return st;
    }
    for (int r = 0; r < S.nrecv; ++r) {
      const long g = S.gi(S.rloc[3 * r], S.rloc[3 * r + 1], S.rloc[3 * r + 2]);
      for (int c = 0; c < 9; ++c)
        S.seis[((size_t)c * S.nrecv + r) * S.d.nt + t] = S.FW[c][g];
    }
    S.steps++;
  }
  return CGFD_OK;
}

template <class R>
void to_vec(std::vector<R> &v, const double *p, long n) {
  v.resize(n);
  for (long q = 0; q < n; ++q) v[q] = (R)p[q];
}
template <class R>
void to_vec(std::vector<R> &v, const float *p, long n) {
  v.resize(n);
  for (long q = 0; q < n; ++q) v[q] = (R)p[q];
}

template <class R>
bool valid_loc(const Solver<R> &S, const int *l) {
  return l[0] >= LFD && l[0] < S.d.ni + LFD && l[1] >= LFD && l[1] < S.d.nj + LFD &&
         l[2] >= LFD && l[2] < S.d.nk + LFD;
}

template <class R>
std::vector<R> *field_set(Solver<R> &S, int set) {
  if (set == CGFD_SET_FW) return S.FW;
  if (set == CGFD_SET_W) return S.W;
  if (set == CGFD_SET_TW) return S.tW;
  return nullptr;
}

}  // namespace

// ------------------------------- C exports ---------------------------------
#define DISPATCH(H, CALL)                                   \
  ((H)->prec == 0 ? CALL(*(Solver<double> *)(H)->s)         \
                  : CALL(*(Solver<float> *)(H)->s))

extern "C" {

int orc_create(const cgfd_desc *d, int prec, void **out) {
  if (!d || !out || (prec != 0 && prec != 1)) return CGFD_ERR_ARG;
  Handle *H = new Handle{prec, nullptr, {}};
  int st;
  if (prec == 0) {
    auto *S = new Solver<double>();
    st = init(*S, *d, g_err);
    H->s = S;
  } else {
    auto *S = new Solver<float>();
    st = init(*S, *d, g_err);
    H->s = S;
  }
  if (st) {
    if (prec == 0) delete (Solver<double> *)H->s; else delete (Solver<float> *)H->s;
    delete H;
    *out = nullptr;
    return st;
  }
  *out = H;
  return CGFD_OK;
}

int orc_destroy(void *h) {
  if (!h) return CGFD_OK;
  Handle *H = (Handle *)h;
  if (H->prec == 0) delete (Solver<double> *)H->s; else delete (Solver<float> *)H->s;
  delete H;
  return CGFD_OK;
}

int orc_last_error(void *h, char *buf, size_t len) {
  const std::string &e = h ? ((Handle *)h)->err : g_err;
  if (buf && len) { std::snprintf(buf, len, "%s", e.c_str()); }
  return CGFD_OK;
}

int orc_upload_metric(void *h, const double *zx, const double *zy, const double *zz,
                      const double *jac) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    to_vec(S.zx, zx, S.N); to_vec(S.zy, zy, S.N); to_vec(S.zz, zz, S.N); to_vec(S.jac, jac, S.N);
    S.have_metric = true; S.prepared = false;
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_upload_media(void *h, const float *alpha, const float *beta, const float *rho) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    to_vec(S.alpha, alpha, S.N); to_vec(S.beta, beta, S.N); to_vec(S.rho, rho, S.N);
    S.have_media = true; S.prepared = false;
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_upload_pml(void *h, const double *apdx, const double *apdy, const double *apdz,
                   const double *bx, const double *by, const double *bz, const double *dbx,
                   const double *dby, const double *dbz) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    to_vec(S.APD[0], apdx, S.nx); to_vec(S.APD[1], apdy, S.ny); to_vec(S.APD[2], apdz, S.nz);
    to_vec(S.B[0], bx, S.nx); to_vec(S.B[1], by, S.ny); to_vec(S.B[2], bz, S.nz);
    to_vec(S.DB[0], dbx, S.nx); to_vec(S.DB[1], dby, S.ny); to_vec(S.DB[2], dbz, S.nz);
    S.have_pml = true; S.prepared = false;
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_upload_moments(void *h, int n, const int *loc, const float *m6, int nstf,
                       const float *stf) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (n < 0 || (n > 0 && (!loc || !m6 || !stf || nstf < 1))) { H->err = "bad moment sources"; return (int)CGFD_ERR_ARG; }
    for (int q = 0; q < n; ++q)
      if (!valid_loc(S, loc + 3 * q)) { H->err = "moment source outside the valid grid"; return (int)CGFD_ERR_ARG; }
    S.nmnt = n; S.nstfm = nstf;
    S.smw[0].clear();
    S.mloc.assign(loc, loc + 3 * n);
    S.m6.assign(m6, m6 + 6 * n);
    S.mstf.assign(stf, stf + (size_t)n * nstf);
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_upload_forces(void *h, int n, const int *loc, const float *f3, int nstf,
                      const float *stf) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (n < 0 || (n > 0 && (!loc || !f3 || !stf || nstf < 1))) { H->err = "bad force sources"; return (int)CGFD_ERR_ARG; }
    for (int q = 0; q < n; ++q)
      if (!valid_loc(S, loc + 3 * q)) { H->err = "force source outside the valid grid"; return (int)CGFD_ERR_ARG; }
    S.nfrc = n; S.nstff = nstf;
    S.smw[1].clear();
    S.floc.assign(loc, loc + 3 * n);
    S.f3.assign(f3, f3 + 3 * n);
    S.fstf.assign(stf, stf + (size_t)n * nstf);
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_upload_focal(void *h, int n, const int *loc, int fnt, double fdt, const float *mom) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (n < 0 || (n > 0 && (!loc || !mom || fnt < 1 || !(fdt > 0)))) { H->err = "bad focal sources"; return (int)CGFD_ERR_ARG; }
    for (int q = 0; q < n; ++q)
      if (!valid_loc(S, loc + 3 * q)) { H->err = "focal source outside the valid grid"; return (int)CGFD_ERR_ARG; }
    S.nfoc = n; S.fnt = fnt; S.fdt = fdt;
    S.smw[2].clear();
    S.focloc.assign(loc, loc + 3 * n);
    S.focmom.assign(mom, mom + (size_t)6 * n * fnt);
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_set_source_smoothing(void *h, int kind, int n, const double *w) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (kind < 0 || kind > 2) { H->err = "bad smoothing kind"; return (int)CGFD_ERR_ARG; }
    const int have = kind == 0 ? S.nmnt : (kind == 1 ? S.nfrc : S.nfoc);
    if (!w || n == 0) {
      S.smw[kind].clear();
      return (int)CGFD_OK;
    }
    if (n != have) { H->err = "smoothing count differs from the sources"; return (int)CGFD_ERR_ARG; }
    S.smw[kind].assign(w, w + (size_t)343 * n);
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_set_receivers(void *h, int n, const int *loc) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (n < 0 || (n > 0 && !loc)) { H->err = "bad receivers"; return (int)CGFD_ERR_ARG; }
    for (int q = 0; q < n; ++q)
      if (!valid_loc(S, loc + 3 * q)) { H->err = "receiver outside the valid grid"; return (int)CGFD_ERR_ARG; }
    S.nrecv = n;
    S.rloc.assign(loc, loc + 3 * n);
    S.seis.assign((size_t)9 * n * S.d.nt, 0.0);
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_rk_stage(void *h, int rk, int curr_t, int X, int Y, int Z) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) { return rk_stage(S, rk, curr_t, X, Y, Z, H->err); };
  return DISPATCH(H, f);
}

int orc_step(void *h, int n) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) { return step(S, n, H->err); };
  return DISPATCH(H, f);
}

int orc_steps_done(void *h, int *n) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) { *n = S.steps; return (int)CGFD_OK; };
  return DISPATCH(H, f);
}

int orc_get_seismograms(void *h, double *out) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    std::memcpy(out, S.seis.data(), S.seis.size() * sizeof(double));
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_get_field(void *h, int set, int comp, double *out) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    auto *fs = field_set(S, set);
    if (!fs || comp < 0 || comp > 8) return (int)CGFD_ERR_ARG;
    for (long q = 0; q < S.N; ++q) out[q] = fs[comp][q];
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

int orc_set_field(void *h, int set, int comp, const double *in) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    auto *fs = field_set(S, set);
    if (!fs || comp < 0 || comp > 8) return (int)CGFD_ERR_ARG;
    for (long q = 0; q < S.N; ++q) fs[comp][q] = in[q];
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

// Auxiliary (ADE) state of one PML direction: set 0 = FA, 1 = A, 2 = tA.
int orc_get_aux(void *h, int dir, int set, int comp, double *out, long *n) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (dir < 0 || dir > 2 || set < 0 || set > 2 || comp < 0 || comp > 8) return (int)CGFD_ERR_ARG;
    auto &v = set == 0 ? S.FA[dir][comp] : (set == 1 ? S.A[dir][comp] : S.tA[dir][comp]);
    *n = (long)v.size();
    if (out) for (size_t q = 0; q < v.size(); ++q) out[q] = v[q];
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

// VelPDcoeff matrices (nx*ny*9 each, reference index (i*ny+j)*9+m).
// Test infrastructure: rounds the stored field sets (mask 1 W, 2 tW, 4 FW) to
// a binary format of ebits/mbits bits with per-component scales (a stored s
// stands for s * scale[c]); flags 1: tW kept as its difference from FW, 2: W
// kept as its difference from FW; adapt >= 0: after every step each scale
// becomes the power of two that puts the component's maximum just below
// 2^adapt; flags 4 (with 1): error feedback -- the last stage keeps the part
// of the new state that FW's rounding drops (r = exact - FW) in the tW set,
// tW = FW + r, and the next step's second stage adds it to the accumulator,
// so FW's roundings do not accumulate in the state; flags 8: every rounding
// stochastic (keyed by step, stage, cell, component and set).  ebits = 0
// turns it off; ebits = 100 + B: block floating point,
// B x-adjacent cells sharing an exponent, mbits magnitude bits each (plus a
// sign).  FP64 oracle only.
int orc_set_storage_emulation(void *h, int ebits, int mbits, const double *scale, int mask,
                              int flags, int adapt) {
  Handle *H = (Handle *)h;
  if (!H || H->prec != 0 || ebits < 0 || (ebits > 11 && ebits < 101) || ebits > 164 ||
      mbits < 1 || mbits > 52 || ((flags & 4) && !(flags & 1)) || ((flags & 8) && ebits >= 100))
    return CGFD_ERR_ARG;
  auto &S = *(Solver<double> *)H->s;
  S.em.ebits = ebits;
  S.em.mbits = mbits;
  S.em.mask = mask;
  S.em.flags = flags;
  S.em.adapt = adapt;
  for (int c = 0; c < 9; ++c) S.em.scale[c] = scale ? scale[c] : 1.0;
  return CGFD_OK;
}

int orc_get_matv(void *h, double *mx, double *my) {
  Handle *H = (Handle *)h;
  auto f = [&](auto &S) {
    if (!(S.have_metric && S.have_media && S.have_pml)) return (int)CGFD_ERR_STATE;
    if (!S.prepared) { vel_pd_coeff(S); S.prepared = true; }
    std::memcpy(mx, S.matVx.data(), S.matVx.size() * sizeof(double));
    std::memcpy(my, S.matVy.data(), S.matVy.size() * sizeof(double));
    return (int)CGFD_OK;
  };
  return DISPATCH(H, f);
}

// ---------------------- host pre-processing restatements --------------------

// gridmesh::calmetric (src/gridmesh.cpp:1476-1627) + common::mirror_extend
// (src/common.cpp:97-135).  out: xi_x xi_y xi_z eta_x eta_y eta_z zeta_x zeta_y
// zeta_z jac; ghost cells not reached by mirror_extend are left at 0.
int orc_metric_from_coords(int ni, int nj, int nk, double steph, const double *x,
                           const double *y, const double *z, double *const out[10]) {
  if (ni < 1 || nj < 1 || nk < 1 || steph <= 0) return CGFD_ERR_ARG;
  const int nx = ni + 6, ny = nj + 6, nz = nk + 6;
  const long N = (long)nx * ny * nz;
  for (int q = 0; q < 10; ++q) std::memset(out[q], 0, N * sizeof(double));
  auto G = [&](int i, int j, int k) { return ((long)i * ny + j) * nz + k; };
#pragma omp parallel for schedule(static)
  for (int i = 3; i < ni + 3; ++i)
    for (int j = 3; j < nj + 3; ++j)
      for (int k = 3; k < nk + 3; ++k) {
        const long g = G(i, j, k);
        const long xp = G(i + 1, j, k), xm = G(i - 1, j, k), yp = G(i, j + 1, k),
                   ym = G(i, j - 1, k), zp = G(i, j, k + 1), zm = G(i, j, k - 1);
        const double v1[3] = {(x[xp] - x[xm]) / 2.0 / steph, (y[xp] - y[xm]) / 2.0 / steph,
                              (z[xp] - z[xm]) / 2.0 / steph};
        const double v2[3] = {(x[yp] - x[ym]) / 2.0 / steph, (y[yp] - y[ym]) / 2.0 / steph,
                              (z[yp] - z[ym]) / 2.0 / steph};
        const double v3[3] = {(x[zp] - x[zm]) / 2.0 / steph, (y[zp] - y[zm]) / 2.0 / steph,
                              (z[zp] - z[zm]) / 2.0 / steph};
        auto cross = [](const double *a, const double *b, double *c) {
          c[0] = a[1] * b[2] - a[2] * b[1];
          c[1] = a[2] * b[0] - a[0] * b[2];
          c[2] = a[0] * b[1] - a[1] * b[0];
        };
        double c12[3], c31[3], c23[3];
        cross(v1, v2, c12);
        cross(v3, v1, c31);
        cross(v2, v3, c23);
        const double J = c12[0] * v3[0] + c12[1] * v3[1] + c12[2] * v3[2];
        out[9][g] = J;
        for (int q = 0; q < 3; ++q) {
          out[6 + q][g] = c12[q] / J;  // zeta
          out[3 + q][g] = c31[q] / J;  // eta
          out[0 + q][g] = c23[q] / J;  // xi
        }
      }
  for (int q = 0; q < 10; ++q) {
    double *v = out[q];
    for (int s = 1; s <= 3; ++s)
      for (int j = 3; j < nj + 3; ++j)
        for (int k = 3; k < nk + 3; ++k) {
          v[G(3 - s, j, k)] = v[G(3 + s, j, k)];
          v[G(ni + 2 + s, j, k)] = v[G(ni + 2 - s, j, k)];
        }
    for (int i = 3; i < ni + 3; ++i)
      for (int k = 3; k < nk + 3; ++k)
        for (int s = 1; s <= 3; ++s) {
          v[G(i, 3 - s, k)] = v[G(i, 3 + s, k)];
          v[G(i, nj + 2 + s, k)] = v[G(i, nj + 2 - s, k)];
        }
    for (int i = 3; i < ni + 3; ++i)
      for (int j = 3; j < nj + 3; ++j)
        for (int s = 1; s <= 3; ++s) {
          v[G(i, j, 3 - s)] = v[G(i, j, 3 + s)];
          v[G(i, j, nk + 2 + s)] = v[G(i, j, nk + 2 - s)];
        }
  }
  return CGFD_OK;
}

// absorb::CalCFSfactors (src/absorb.cpp:346-805) with PD=2, PB=2, PA=1.
int orc_cfs_factors(int ni, int nj, int nk, const int *nabs, const double *velabs,
                    const double *bmax, const double *amax, const double *dlx,
                    const double *dly, const double *dlz, double *apdx, double *apdy,
                    double *apdz, double *bx, double *by, double *bz, double *dbx,
                    double *dby, double *dbz) {
  const int n3[3] = {ni + 6, nj + 6, nk + 6};
  const int nv[3] = {ni, nj, nk};
  const double *dl[3] = {dlx, dly, dlz};
  double *apd[3] = {apdx, apdy, apdz}, *bb[3] = {bx, by, bz}, *db[3] = {dbx, dby, dbz};
  const double PD = 2.0, PB = 2.0, PA = 1.0;
  for (int a = 0; a < 3; ++a) {
    const int n = n3[a];
    std::vector<double> Af(n, 0.0), Bf(n, 1.0), Df(n, 0.0), L(n + 1, 0.0);
    for (int side = 0; side < 2; ++side) {
      const int q = 2 * a + side;
      const int w = nabs[q];
      if (w <= 0) continue;
      const double Rpp = std::pow(10.0, -(std::log10(w * 1.0) - 1) / std::log10(2.0) - 3.0);
      int lo, hi;
      double L0;
      if (side == 0) {  // X1: accumulate from the inner edge outwards
        lo = 3; hi = 3 + w - 1;
        for (int i = hi; i >= lo; --i) L[i] = L[i + 1] + dl[a][i];
        L0 = L[lo];
      } else {          // X2
        lo = 3 + nv[a] - w; hi = 3 + nv[a] - 1;
        for (int i = lo; i <= hi; ++i) L[i] = L[i - 1] + dl[a][i];
        L0 = L[hi];
      }
      const double dmax = -velabs[q] / 2.0 / L0 * std::log(Rpp) * (PD + 1.0);
      for (int i = lo; i <= hi; ++i) {
        if (L[i] < 0) { Df[i] = 0; Bf[i] = 1; Af[i] = 0; continue; }
        Df[i] = dmax * std::pow(L[i] / L0, PD);
        Bf[i] = 1.0 + (bmax[q] - 1.0) * std::pow(L[i] / L0, PB);
        Af[i] = amax[q] * (1.0 - std::pow(L[i] / L0, PA));
      }
    }
    for (int i = 0; i < n; ++i) {
      bb[a][i] = Bf[i];
      apd[a][i] = Af[i] + Df[i] / Bf[i];
      db[a][i] = Df[i] / Bf[i];
    }
  }
  return CGFD_OK;
}

// Wavelets of src/mathfunc.cpp:481-608 sampled as source::cal_stf_moment.
int orc_stf(int type, double start, double t0, double f0, int n, double dt, double *out) {
  const double PI = 3.141592653589793, ZERO = 1.e-20;
  for (int i = 0; i < n; ++i) {
    const double t = i * dt - start;
    double s = 0;
    switch (type) {
      case CGFD_STF_GAUSS:
        s = (std::fabs(t0) >= ZERO && (t <= 0.0 || t >= 2.0 * t0)) ? 0.0
            : std::exp(-(t - t0) * (t - t0) / (f0 * f0)) / (std::sqrt(PI) * f0);
        break;
      case CGFD_STF_GAUSS_D:
        s = (std::fabs(t0) >= ZERO && (t <= 0.0 || t >= 2.0 * t0)) ? 0.0
            : std::exp(-(t - t0) * (t - t0) / (f0 * f0)) / (std::sqrt(PI) * f0) *
                  (-2.0 * (t - t0) / (f0 * f0));
        break;
      case CGFD_STF_RICKER:
        if (t > 0.0) {
          const double u = (t - t0) * 2.0 * PI * f0;
          s = (u * u / 4.0 - 0.5) * std::exp(-u * u / 4.0) * std::sqrt(PI) / 2.0;
        }
        break;
      case CGFD_STF_RICKER_D:
        if (t > 0.0) {
          const double u = (t - t0) * 2.0 * PI * f0;
          s = u * (1.5 - u * u / 4.0) * std::exp(-u * u / 4.0) * std::sqrt(PI) / 2.0 * PI * f0;
        }
        break;
      case CGFD_STF_BELL: {
        const double x = t - t0;
        s = (x > 0.0 && x < f0) ? (1.0 - std::cos(2.0 * PI * x / f0)) / f0 : 0.0;
      } break;
      case CGFD_STF_BELL_D: {
        const double x = t - t0;
        s = (x > 0.0 && x < f0) ? 2.0 * PI * std::sin(2.0 * PI * x / f0) / f0 : 0.0;
      } break;
      case CGFD_STF_BELL_I: {
        const double x = t - t0;
        s = x <= 0.0 ? 0.0 : (x < f0 ? x / f0 - std::sin(2.0 * PI * x / f0) / (2.0 * PI) : 1.0);
      } break;
      case CGFD_STF_STEP:
        s = t > 0.0 ? 1.0 : 0.0;
        break;
      default:
        return CGFD_ERR_ARG;
    }
    out[i] = std::fabs(s) < ZERO ? 0.0 : s;
  }
  return CGFD_OK;
}

// source::angle2moment (src/source.cpp:134-155).
int orc_angle2moment(double strike, double dip, double rake, double *m6) {
  const double PI = 3.141592653589793;
  const double S = strike / 180.0 * PI, D = dip / 180.0 * PI, R = rake / 180.0 * PI;
  const double m11 = -(std::sin(D) * std::cos(R) * std::sin(2.0 * S) +
                       std::sin(2.0 * D) * std::sin(R) * std::sin(S) * std::sin(S));
  const double m22 = std::sin(D) * std::cos(R) * std::sin(2.0 * S) -
                     std::sin(2.0 * D) * std::sin(R) * std::cos(S) * std::cos(S);
  m6[0] = m11;
  m6[1] = m22;
  m6[2] = -(m11 + m22);
  m6[3] = std::sin(D) * std::cos(R) * std::cos(2.0 * S) +
          std::sin(2.0 * D) * std::sin(R) * std::sin(2.0 * S) * 0.5;
  m6[4] = -(std::cos(D) * std::cos(R) * std::cos(S) + std::cos(2.0 * D) * std::sin(R) * std::sin(S));
  m6[5] = -(std::cos(D) * std::cos(R) * std::sin(S) - std::cos(2.0 * D) * std::sin(R) * std::cos(S));
  return CGFD_OK;
}

}  // extern "C"
