// setup.cpp -- host pre-processing in FP64 that feeds the solver: grid
// metric from node coordinates, ADE CFS-PML profiles, source time functions
// and the strike/dip/rake moment tensor.
//
// These replace the rank-0 pre-processing of the reference:
//   gridmesh::calmetric      src/gridmesh.cpp:1476-1627 (+ common::mirror_extend,
//                            src/common.cpp:97-135)
//   absorb::CalCFSfactors    src/absorb.cpp:346-805
//   mathfunc wavelets        src/mathfunc.cpp:481-608, sampled like
//                            source::cal_stf_moment (src/source.cpp:102-131)
//   source::angle2moment     src/source.cpp:134-155
#include "../../include/cgfd.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr double kPi = 3.141592653589793;

struct Dims {
  int nx, ny, nz;
  long at(int i, int j, int k) const { return ((long)i * ny + j) * nz + k; }
};

// Copies valid-cell values into the 3 ghost layers of each face, one axis at
// a time and only across the valid range of the other two axes (so edges and
// corners are not filled), as common::mirror_extend does.
void mirror_ghosts(double *v, const Dims &D, int ni, int nj, int nk) {
  for (int s = 1; s <= 3; ++s)
    for (int j = 3; j < nj + 3; ++j)
      for (int k = 3; k < nk + 3; ++k) {
        v[D.at(3 - s, j, k)] = v[D.at(3 + s, j, k)];
        v[D.at(ni + 2 + s, j, k)] = v[D.at(ni + 2 - s, j, k)];
      }
  for (int s = 1; s <= 3; ++s)
    for (int i = 3; i < ni + 3; ++i)
      for (int k = 3; k < nk + 3; ++k) {
        v[D.at(i, 3 - s, k)] = v[D.at(i, 3 + s, k)];
        v[D.at(i, nj + 2 + s, k)] = v[D.at(i, nj + 2 - s, k)];
      }
  for (int s = 1; s <= 3; ++s)
    for (int i = 3; i < ni + 3; ++i)
      for (int j = 3; j < nj + 3; ++j) {
        v[D.at(i, j, 3 - s)] = v[D.at(i, j, 3 + s)];
        v[D.at(i, j, nk + 2 + s)] = v[D.at(i, j, nk + 2 - s)];
      }
}

}  // namespace

extern "C" {

int cgfd_metric_from_coords(int ni, int nj, int nk, double steph, const double *x,
                            const double *y, const double *z, double *const out[10]) {
  if (ni < 1 || nj < 1 || nk < 1 || !(steph > 0) || !x || !y || !z || !out)
    return CGFD_ERR_ARG;
  for (int q = 0; q < 10; ++q)
    if (!out[q]) return CGFD_ERR_ARG;
  const Dims D{ni + 6, nj + 6, nk + 6};
  const long n = (long)D.nx * D.ny * D.nz;
  for (int q = 0; q < 10; ++q) std::memset(out[q], 0, n * sizeof(double));
  const double s2 = 2.0 * steph;
  for (int i = 3; i < ni + 3; ++i)
    for (int j = 3; j < nj + 3; ++j)
      for (int k = 3; k < nk + 3; ++k) {
        const long c = D.at(i, j, k);
        // covariant basis r_xi, r_eta, r_zeta by 2-point central differences,
        // normalised by steph (the metric is that of the index grid times h)
        const long nb[3][2] = {{D.at(i + 1, j, k), D.at(i - 1, j, k)},
                               {D.at(i, j + 1, k), D.at(i, j - 1, k)},
                               {D.at(i, j, k + 1), D.at(i, j, k - 1)}};
        double r[3][3];
        for (int a = 0; a < 3; ++a) {
          r[a][0] = (x[nb[a][0]] - x[nb[a][1]]) / s2;
          r[a][1] = (y[nb[a][0]] - y[nb[a][1]]) / s2;
          r[a][2] = (z[nb[a][0]] - z[nb[a][1]]) / s2;
        }
        // contravariant basis = cross products of the other two / J
        double g[3][3];
        for (int a = 0; a < 3; ++a) {
          const double *p = r[(a + 1) % 3], *q = r[(a + 2) % 3];
          g[a][0] = p[1] * q[2] - p[2] * q[1];
          g[a][1] = p[2] * q[0] - p[0] * q[2];
          g[a][2] = p[0] * q[1] - p[1] * q[0];
        }
        const double J = g[2][0] * r[2][0] + g[2][1] * r[2][1] + g[2][2] * r[2][2];
        out[9][c] = J;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) out[3 * a + b][c] = g[a][b] / J;
      }
  for (int q = 0; q < 10; ++q) mirror_ghosts(out[q], D, ni, nj, nk);
  return CGFD_OK;
}

int cgfd_cfs_factors(int ni, int nj, int nk, const int nabs[6], const double velabs[6],
                     const double bmax[6], const double amax[6], const double *dlx,
                     const double *dly, const double *dlz, double *apd_x, double *apd_y,
                     double *apd_z, double *b_x, double *b_y, double *b_z, double *db_x,
                     double *db_y, double *db_z) {
  if (ni < 1 || nj < 1 || nk < 1 || !nabs || !velabs || !bmax || !amax || !dlx || !dly ||
      !dlz || !apd_x || !apd_y || !apd_z || !b_x || !b_y || !b_z || !db_x || !db_y || !db_z)
    return CGFD_ERR_ARG;
  const int nvalid[3] = {ni, nj, nk};
  const double *dl[3] = {dlx, dly, dlz};
  double *apd[3] = {apd_x, apd_y, apd_z}, *bb[3] = {b_x, b_y, b_z}, *db[3] = {db_x, db_y, db_z};
  // exponents of the d, beta and alpha profiles (Zhang 2010 ADE CFS-PML)
  const double PD = 2.0, PB = 2.0, PA = 1.0;
  for (int ax = 0; ax < 3; ++ax) {
    const int n = nvalid[ax] + 6;
    std::vector<double> alpha(n, 0.0), beta(n, 1.0), d(n, 0.0);
    // distance into the layer measured from its inner edge, one cell-width
    // per cell; both faces share this array, so a face that touches the other
    // face's layer continues its distance (the reference does the same)
    std::vector<double> L(n + 1, 0.0);
    for (int side = 0; side < 2; ++side) {
      const int face = 2 * ax + side, w = nabs[face];
      if (w < 1) continue;
      int lo, hi;
      if (side == 0) {
        lo = 3;
        hi = 3 + w - 1;
        for (int c = hi; c >= lo; --c) L[c] = L[c + 1] + dl[ax][c];
      } else {
        lo = nvalid[ax] + 3 - w;
        hi = nvalid[ax] + 2;
        for (int c = lo; c <= hi; ++c) L[c] = L[c - 1] + dl[ax][c];
      }
      const double L0 = side == 0 ? L[lo] : L[hi];
      // theoretical reflection coefficient and peak damping
      const double R = std::pow(10.0, -(std::log10((double)w) - 1.0) / std::log10(2.0) - 3.0);
      const double dmax = -velabs[face] / 2.0 / L0 * std::log(R) * (PD + 1.0);
      for (int c = lo; c <= hi; ++c) {
        if (L[c] < 0) continue;
        const double r = L[c] / L0;
        d[c] = dmax * std::pow(r, PD);
        beta[c] = 1.0 + (bmax[face] - 1.0) * std::pow(r, PB);
        alpha[c] = amax[face] * (1.0 - std::pow(r, PA));
      }
    }
    for (int c = 0; c < n; ++c) {
      bb[ax][c] = beta[c];
      db[ax][c] = d[c] / beta[c];
      apd[ax][c] = alpha[c] + d[c] / beta[c];
    }
  }
  return CGFD_OK;
}

int cgfd_stf(int type, double start, double t0, double f0, int n, double dt, float *out) {
  if (n < 0 || (n > 0 && !out)) return CGFD_ERR_ARG;
  if (type < CGFD_STF_GAUSS || type > CGFD_STF_STEP) return CGFD_ERR_ARG;
  for (int q = 0; q < n; ++q) {
    const double t = q * dt - start;
    double v = 0.0;
    if (type == CGFD_STF_GAUSS || type == CGFD_STF_GAUSS_D) {
      // Gaussian of width f0 centred on t0, cut outside (0, 2 t0)
      const bool cut = std::fabs(t0) >= 1e-20 && (t <= 0.0 || t >= 2.0 * t0);
      if (!cut) {
        v = std::exp(-(t - t0) * (t - t0) / (f0 * f0)) / (std::sqrt(kPi) * f0);
        if (type == CGFD_STF_GAUSS_D) v *= -2.0 * (t - t0) / (f0 * f0);
      }
    } else if (type == CGFD_STF_RICKER || type == CGFD_STF_RICKER_D) {
      if (t > 0.0) {
        const double u = (t - t0) * 2.0 * kPi * f0, e = std::exp(-u * u / 4.0);
        v = type == CGFD_STF_RICKER ? (u * u / 4.0 - 0.5) * e * std::sqrt(kPi) / 2.0
                                    : u * (1.5 - u * u / 4.0) * e * std::sqrt(kPi) / 2.0 * kPi * f0;
      }
    } else if (type == CGFD_STF_STEP) {
      v = t > 0.0 ? 1.0 : 0.0;
    } else {  // bell family, shifted by t0, width f0
      const double s = t - t0, w = f0;
      if (type == CGFD_STF_BELL) v = (s > 0.0 && s < w) ? (1.0 - std::cos(2.0 * kPi * s / w)) / w : 0.0;
      else if (type == CGFD_STF_BELL_D) v = (s > 0.0 && s < w) ? 2.0 * kPi * std::sin(2.0 * kPi * s / w) / w : 0.0;
      else v = s <= 0.0 ? 0.0 : (s < w ? s / w - std::sin(2.0 * kPi * s / w) / (2.0 * kPi) : 1.0);
    }
    out[q] = std::fabs(v) < 1e-20 ? 0.f : (float)v;
  }
  return CGFD_OK;
}

int cgfd_angle2moment(double strike, double dip, double rake, double m6[6]) {
  if (!m6) return CGFD_ERR_ARG;
  const double s = strike * kPi / 180.0, d = dip * kPi / 180.0, r = rake * kPi / 180.0;
  const double sd = std::sin(d), cd = std::cos(d), s2d = std::sin(2 * d), c2d = std::cos(2 * d);
  const double sr = std::sin(r), cr = std::cos(r);
  const double ss = std::sin(s), cs = std::cos(s), s2s = std::sin(2 * s), c2s = std::cos(2 * s);
  // Aki & Richards convention (x north, y east, z down as in the reference)
  const double mxx = -(sd * cr * s2s + s2d * sr * ss * ss);
  const double myy = sd * cr * s2s - s2d * sr * cs * cs;
  m6[0] = mxx;
  m6[1] = myy;
  m6[2] = -(mxx + myy);
  m6[3] = sd * cr * c2s + 0.5 * s2d * sr * s2s;
  m6[4] = -(cd * cr * cs + c2d * sr * ss);
  m6[5] = -(cd * cr * ss - c2d * sr * cs);
  return CGFD_OK;
}

}  // extern "C"
