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
//   gridmesh::read_vmapnew   src/gridmesh.cpp:72-533 (+ smooth_zdepth and
//                            set_twoside_space 1092-1210, and the ghost
//                            extension common::interpolated_extend,
//                            src/common.cpp:67-130)
//   common::reposition       src/common.cpp:225-270 (source and receiver
//                            location, src/source.cpp:985-1300 and
//                            src/seisplot.cpp:412-426)
//   source smoothing         src/source.cpp:157-378 (MomentShiftPosition,
//                            eighth_locate, cal_norm; the SrcSmooth build)
#include "../../include/cgfd.h"
#include "abi_guard.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace cgfd {
void set_global_error(const char *msg);
}

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

// ---------------------------- vmap grid -----------------------------------

// The spacing pair (ha0, hb0) of the two constant-spacing ends of a graded
// layer: na intervals next to the layer above within [ha1, ha2], nb next to
// the layer below within [hb1, hb2], together of length l; the free length
// is shared in proportion to the two ranges (set_twoside_space).
void two_sided_spacing(double l, int na, int nb, double ha1, double ha2, double hb1, double hb2,
                       double *ha0, double *hb0) {
  const double free_len = l - na * ha1 - nb * hb1;
  const double ra = na * (ha2 - ha1), rb = nb * (hb2 - hb1);
  const double eps = 1.e-5;
  if (std::fabs(free_len) < eps) {
    *ha0 = ha1;
    *hb0 = hb1;
  } else if (std::fabs(ra) < eps) {
    *ha0 = ha1;
    *hb0 = hb1 + free_len / nb;
  } else if (std::fabs(rb) < eps) {
    *ha0 = ha1 + free_len / na;
    *hb0 = hb1;
  } else {
    *ha0 = ha1 + free_len * ra / (ra + rb) / na;
    *hb0 = hb1 + free_len * rb / (ra + rb) / nb;
  }
}

// Node depths z[0..n] (bottom zb to top za) of a layer of n intervals whose
// spacing grades from hb (the layer below) to ha (the layer above)
// (smooth_zdepth).  When the mean spacing lies between ha and hb, a
// geometric run of intervals between constant ends, the run shortened one
// interval at a time until the ends can take up the remaining length;
// otherwise linear ramps over a quarter of the intervals at each end around
// a constant middle.  False where the reference's search would not end.
bool graded_layer(double za, double zb, double ha, double hb, int n, double *z) {
  if (n < 1) return false;
  std::vector<double> h(n + 2);
  const double l = za - zb, h0 = l / n;
  h[0] = hb;
  h[n + 1] = ha;
  if ((h0 >= ha && h0 <= hb) || (h0 <= ha && h0 >= hb)) {
    int nb = 1, na = n, n0 = n;
    for (;;) {
      if (n0 < 0) return false;
      double run = 0.0;
      const double f = std::pow(ha / hb, 1.0 / (n0 + 1)) - 1.0;
      for (int k = 1; k <= nb - 1; ++k) h[k] = hb;
      for (int k = na + 1; k <= n + 1; ++k) h[k] = ha;
      for (int k = nb; k <= na; ++k) {
        h[k] = h[k - 1] * (1 + f);
        run += h[k];
      }
      const double ha1 = ha * std::min(1.0, 1.0 - f), ha2 = ha * std::max(1.0, 1.0 - f);
      const double hb1 = hb * std::min(1.0, 1.0 + f), hb2 = hb * std::max(1.0, 1.0 + f);
      const double la1 = (n - na) * ha1, la2 = (n - na) * ha2;
      const double lb1 = (nb - 1) * hb1, lb2 = (nb - 1) * hb2;
      if ((la1 + lb1 <= l - run) && (l - run <= la2 + lb2)) {
        double ha0, hb0;
        two_sided_spacing(l - run, n - na, nb - 1, ha1, ha2, hb1, hb2, &ha0, &hb0);
        for (int k = na + 1; k <= n; ++k) h[k] = ha0;
        for (int k = 1; k <= nb - 1; ++k) h[k] = hb0;
        break;
      }
      // the ends are too long (or too short) for the rest: hand one interval
      // of the run to the end with the smaller (or larger) spacing
      const bool too_long = l - run < la1 + lb1;
      if (too_long == (ha < hb)) --na;
      else ++nb;
      --n0;
    }
  } else {
    const int na = n / 4, nb = n / 4, n0 = n - na - nb;
    if (nb < 1) return false;
    const double la1 = (na + 1) * na / 2.0, lb1 = (nb + 1) * nb / 2.0;
    const double la2 = la1 + na * lb1 / nb + na * n0;
    const double l0 = l - na * ha - nb * hb - n0 * ha - la1 * (ha - hb) / nb;
    const double ha0 = l0 / la2, hb0 = (na * ha0 + ha - hb) / nb;
    for (int k = 1; k <= nb; ++k) h[k] = hb + k * hb0;
    for (int k = nb + 1; k <= nb + n0; ++k) h[k] = h[k - 1];
    for (int k = nb + n0 + 1; k <= n; ++k) h[k] = ha + (n - k + 1) * ha0;
  }
  z[0] = 0.0;
  for (int k = 0; k < n; ++k) z[k + 1] = z[k] + h[k + 1];
  for (int k = 0; k < n + 1; ++k) z[k] = z[k] + zb;
  return true;
}

// Ghost nodes by linear extrapolation 2 v[edge] - v[edge -+ s], along z for
// every (x, y) column, then y, then x over the whole array (edges and
// corners included), as common::interpolated_extend.
void extend_linear(double *v, const Dims &D, int ni, int nj, int nk) {
  for (int i = 0; i < D.nx; ++i)
    for (int j = 0; j < D.ny; ++j)
      for (int s = 1; s <= 3; ++s) {
        v[D.at(i, j, 3 - s)] = 2.0 * v[D.at(i, j, 3)] - v[D.at(i, j, 3 + s)];
        v[D.at(i, j, nk + 2 + s)] = 2.0 * v[D.at(i, j, nk + 2)] - v[D.at(i, j, nk + 2 - s)];
      }
  for (int i = 0; i < D.nx; ++i)
    for (int k = 0; k < D.nz; ++k)
      for (int s = 1; s <= 3; ++s) {
        v[D.at(i, 3 - s, k)] = 2.0 * v[D.at(i, 3, k)] - v[D.at(i, 3 + s, k)];
        v[D.at(i, nj + 2 + s, k)] = 2.0 * v[D.at(i, nj + 2, k)] - v[D.at(i, nj + 2 - s, k)];
      }
  for (int j = 0; j < D.ny; ++j)
    for (int k = 0; k < D.nz; ++k)
      for (int s = 1; s <= 3; ++s) {
        v[D.at(3 - s, j, k)] = 2.0 * v[D.at(3, j, k)] - v[D.at(3 + s, j, k)];
        v[D.at(ni + 2 + s, j, k)] = 2.0 * v[D.at(ni + 2, j, k)] - v[D.at(ni + 2 - s, j, k)];
      }
}

// ---------------------------- volume media ---------------------------------

// Bracketing samples of v on an increasing axis a[0..n-1]: (L, R) and the
// value to interpolate at, clamped to the axis ends (mathfunc::LocValue1d).
void bracket(double v, const double *a, int n, int *L, int *R, double *at) {
  *L = 0;
  *R = n - 1;
  *at = v;
  if (v <= a[0]) {
    *at = a[0];
    *R = 1;
  } else if (v >= a[n - 1]) {
    *at = a[n - 1];
    *L = n - 2;
  } else {
    while (*R - *L > 1) {
      const int m = (*R - *L) / 2 + *L;
      if (a[m] == v) {
        *L = m;
        *R = m + 1;
        break;
      }
      if (a[m] > v) *R = m;
      else *L = m;
    }
  }
}

// Lagrange weights of the n nodes X at x0, products taken as
// mathfunc::interp3d takes them
void lagrange(const double *X, int n, double x0, double *w) {
  for (int i = 0; i < n; ++i) {
    w[i] = 1.0;
    for (int j = 0; j < n; ++j)
      if (j != i) w[i] *= (X[j] - x0) / (X[j] - X[i]);
  }
}

struct Volume {
  const double *x, *y, *z;  // the axes of the selected sub-volume
  int nx, ny, nz;
  const float *vp, *vs, *rho;  // full volume [nvx][nvy][nvz]
  int x0, y0, z0, nvy, nvz;     // sub-volume origin, full strides
  // Vp, Vs, density at a point (mediapar::volume_discrete): trilinear
  // between the bracketing samples, the point clamped to the sub-volume
  void at(double px, double py, double pz, double *vpo, double *vso, double *dco) const {
    int i1, i2, j1, j2, k1, k2;
    double qx, qy, qz;
    bracket(px, x, nx, &i1, &i2, &qx);
    bracket(py, y, ny, &j1, &j2, &qy);
    bracket(pz, z, nz, &k1, &k2, &qz);
    const double X[2] = {x[i1], x[i1 + 1]}, Y[2] = {y[j1], y[j1 + 1]}, Z[2] = {z[k1], z[k1 + 1]};
    double wx[2], wy[2], wz[2];
    lagrange(X, 2, qx, wx);
    lagrange(Y, 2, qy, wy);
    lagrange(Z, 2, qz, wz);
    const float *src[3] = {vp, vs, rho};
    double *dst[3] = {vpo, vso, dco};
    for (int q = 0; q < 3; ++q) {
      double f = 0.0;
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int c = 0; c < 2; ++c)
            f += wx[a] * wy[b] * wz[c] *
                 (double)src[q][((size_t)(x0 + i1 + a) * nvy + (y0 + j1 + b)) * nvz + (z0 + k1 + c)];
      *dst[q] = f;
    }
  }
};

int grid_fail(const std::string &msg) {
  cgfd::set_global_error(("cgfd_grid_vmap: " + msg).c_str());
  return CGFD_ERR_ARG;
}

}  // namespace

extern "C" {

int cgfd_metric_from_coords(int ni, int nj, int nk, double steph, const double *x,
                            const double *y, const double *z, double *const out[10]) {
  CGFD_ABI_BEGIN
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
  CGFD_ABI_END(nullptr)
}

int cgfd_cfs_factors(int ni, int nj, int nk, const int nabs[6], const double velabs[6],
                     const double bmax[6], const double amax[6], const double *dlx,
                     const double *dly, const double *dlz, double *apd_x, double *apd_y,
                     double *apd_z, double *b_x, double *b_y, double *b_z, double *db_x,
                     double *db_y, double *db_z) {
  CGFD_ABI_BEGIN
  if (ni < 1 || nj < 1 || nk < 1 || !nabs || !velabs || !bmax || !amax || !dlx || !dly ||
      !dlz || !apd_x || !apd_y || !apd_z || !b_x || !b_y || !b_z || !db_x || !db_y || !db_z)
    return CGFD_ERR_ARG;
  const int nvalid[3] = {ni, nj, nk};
  for (int face = 0; face < 6; ++face)
    if (nabs[face] < 0 || nabs[face] > nvalid[face / 2]) {
      cgfd::set_global_error(
          "cgfd_cfs_factors: a layer is of negative width or wider than the grid along its axis");
      return CGFD_ERR_ARG;
    }
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
  CGFD_ABI_END(nullptr)
}

int cgfd_stf(int type, double start, double t0, double f0, int n, double dt, float *out) {
  CGFD_ABI_BEGIN
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
  CGFD_ABI_END(nullptr)
}

int cgfd_angle2moment(double strike, double dip, double rake, double m6[6]) {
  CGFD_ABI_BEGIN
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
  CGFD_ABI_END(nullptr)
}

int cgfd_grid_vmap(int ni, int nj, int nk, int nsurf, const int *gridpoints,
                   const int *equalspacing, const double *anchor, int hybrid,
                   double convers_depth, double *x, double *y, double *z, int *con_index) {
  CGFD_ABI_BEGIN
  if (ni < 1 || nj < 1 || nk < 2 || nsurf < 2 || !gridpoints || !equalspacing || !anchor || !x ||
      !y || !z || !con_index)
    return grid_fail("bad arguments");
  const int nl = nsurf - 1;  // layers
  const Dims D{ni + 6, nj + 6, nk + 6};
  const int stride = 2 + nsurf;  // per column: x, y, z_0 .. z_{nsurf-1}
  auto col = [&](int i, int j) { return anchor + ((size_t)i * nj + j) * stride; };
  // the reference's checks (src/gridmesh.cpp:134-158)
  long total = 0;
  for (int l = 0; l < nl; ++l) {
    if (gridpoints[l] < 1) return grid_fail("every layer needs at least one interval");
    total += gridpoints[l];
  }
  if (!equalspacing[0] || !equalspacing[nl - 1])
    return grid_fail("the first and the last layer must be equally spaced");
  for (int l = 1; l < nl; ++l)
    if (!equalspacing[l - 1] && !equalspacing[l])
      return grid_fail("two adjacent layers cannot both be graded");
  if (total + 1 != nk) return grid_fail("the layers' intervals + 1 must equal nk");
  for (int i = 0; i < ni; ++i)
    for (int j = 0; j < nj; ++j) {
      for (int q = 0; q < stride; ++q)
        if (!std::isfinite(col(i, j)[q])) return grid_fail("anchor values must be finite");
      for (int q = 1; q < nsurf; ++q)
        if (col(i, j)[2 + q] > col(i, j)[1 + q])
          return grid_fail("interface depths must decrease from the top down");
    }

  // the layer stack actually meshed: the given one, or (hybrid) its layers
  // above the conversion depth, the layer holding it cut there, and one flat
  // layer from there to the deepest point of the last interface, the nk - 1
  // intervals shared in proportion to the layers' thickness ranges
  std::vector<int> gp(gridpoints, gridpoints + nl);
  std::vector<int> eq(equalspacing, equalspacing + nl);
  int ns = nsurf;           // interfaces meshed
  double z_conv = 0, z_bottom = 0;
  int conv_iface = -1;      // hybrid: index of the conversion interface
  if (hybrid) {
    std::vector<double> iface_min(nsurf), iface_max(nsurf), layer_min(nl), layer_max(nl);
    for (int q = 0; q < nsurf; ++q) {
      iface_min[q] = iface_max[q] = col(0, 0)[2 + q];
      for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j) {
          iface_min[q] = std::min(iface_min[q], col(i, j)[2 + q]);
          iface_max[q] = std::max(iface_max[q], col(i, j)[2 + q]);
        }
    }
    for (int l = 0; l < nl; ++l) {  // [lowest bottom, highest top]
      layer_max[l] = iface_max[l];
      layer_min[l] = iface_min[l + 1];
    }
    for (int l = 0; l < nl; ++l)
      if (convers_depth >= layer_min[l] && convers_depth <= layer_max[l]) {
        conv_iface = l + 1;
        break;
      }
    if (conv_iface < 0) return grid_fail("the conversion depth lies in no layer");
    z_conv = convers_depth;
    z_bottom = iface_min[nsurf - 1];
    ns = conv_iface + 2;
    // thickness ranges of the new layers
    std::vector<double> lo(conv_iface + 1), hi(conv_iface + 1);
    for (int l = 0; l < conv_iface; ++l) {
      lo[l] = layer_min[l];
      hi[l] = layer_max[l];
    }
    lo[conv_iface - 1] = z_conv;
    lo[conv_iface] = z_bottom;
    hi[conv_iface] = z_conv;
    double total_len = 0;
    for (int l = 0; l <= conv_iface; ++l) total_len += hi[l] - lo[l];
    gp.assign(conv_iface + 1, 0);
    eq.assign(conv_iface + 1, 1);
    for (int l = 0; l < conv_iface; ++l) eq[l] = equalspacing[l];
    gp[conv_iface] = nk - 1;
    for (int l = 0; l < conv_iface; ++l) {
      const double share = nk * (hi[l] - lo[l]) / total_len;  // truncated, as the reference
      if (!(share >= 0.0 && share <= nk))
        return grid_fail("the hybrid grid's layer thicknesses give no valid split");
      gp[l] = (int)share;
      gp[conv_iface] -= gp[l];
    }
    for (int l = 0; l <= conv_iface; ++l)
      if (gp[l] < 1) return grid_fail("a layer of the hybrid grid receives no interval");
  }
  // node index of each interface: the last at the bottom (3), upwards from there
  std::vector<int> kidx(ns);
  kidx[ns - 1] = 3;
  for (int q = ns - 2; q >= 0; --q) kidx[q] = kidx[q + 1] + gp[q];
  *con_index = hybrid ? kidx[ns - 1] + gp[ns - 2] : 3;

  std::vector<double> zi(ns), zv(D.nz);
  for (int i = 0; i < ni; ++i)
    for (int j = 0; j < nj; ++j) {
      const double *c = col(i, j);
      for (int q = 0; q < ns; ++q)
        zi[q] = !hybrid || q < conv_iface ? c[2 + q] : (q == conv_iface ? z_conv : z_bottom);
      for (int l = 0; l < ns - 1; ++l) {
        const int top = kidx[l], bot = kidx[l + 1];
        if (eq[l]) {
          const double step = (zi[l] - zi[l + 1]) / (1.0 * gp[l]);
          for (int m = bot; m <= top; ++m) zv[m] = zi[l] + (m - top) * step;
        } else {
          const double ha = (zi[l - 1] - zi[l]) / (1.0 * gp[l - 1]);
          const double hb = (zi[l + 1] - zi[l + 2]) / (1.0 * gp[l + 1]);
          if (!graded_layer(zi[l], zi[l + 1], ha, hb, gp[l], &zv[bot]))
            return grid_fail("a graded layer cannot join its neighbours' spacings");
        }
        zv[top] = zi[l];
        zv[bot] = zi[l + 1];
      }
      for (int k = 3; k < nk + 3; ++k) {
        const long g = D.at(i + 3, j + 3, k);
        x[g] = c[0];
        y[g] = c[1];
        z[g] = zv[k];
      }
    }
  extend_linear(x, D, ni, nj, nk);
  extend_linear(y, D, ni, nj, nk);
  extend_linear(z, D, ni, nj, nk);
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

int cgfd_media_volume(int ni, int nj, int nk, const double *x, const double *y, const double *z,
                      int nvx, int nvy, int nvz, const double *vx, const double *vy,
                      const double *vz, const float *vp, const float *vs, const float *rho,
                      double crit_value, double crit_perc, int sampx, int sampy, int sampz,
                      float *alpha, float *beta, float *dens) {
  CGFD_ABI_BEGIN
  auto fail = [](const char *m) {
    cgfd::set_global_error((std::string("cgfd_media_volume: ") + m).c_str());
    return CGFD_ERR_ARG;
  };
  if (ni < 1 || nj < 1 || nk < 1 || !x || !y || !z || nvx < 2 || nvy < 2 || nvz < 2 || !vx ||
      !vy || !vz || !vp || !vs || !rho || sampx < 1 || sampy < 1 || sampz < 1 || !alpha ||
      !beta || !dens)
    return fail("bad arguments");
  const double *ax[3] = {vx, vy, vz};
  const int na[3] = {nvx, nvy, nvz};
  for (int d = 0; d < 3; ++d)
    for (int q = 1; q < na[d]; ++q)
      if (!(ax[d][q] > ax[d][q - 1])) return fail("volume axes must increase");
  const Dims D{ni + 6, nj + 6, nk + 6};
  // the sub-volume that brackets the valid nodes (mediapar::read_volume_new)
  const double *cc[3] = {x, y, z};
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    double mn = cc[d][D.at(3, 3, 3)], mx = mn;
    for (int i = 3; i < ni + 3; ++i)
      for (int j = 3; j < nj + 3; ++j)
        for (int k = 3; k < nk + 3; ++k) {
          mn = std::min(mn, cc[d][D.at(i, j, k)]);
          mx = std::max(mx, cc[d][D.at(i, j, k)]);
        }
    int L, R;
    double v;
    bracket(mn, ax[d], na[d], &L, &R, &v);
    lo[d] = L;
    bracket(mx, ax[d], na[d], &L, &R, &v);
    hi[d] = R;
  }
  const Volume V{vx + lo[0], vy + lo[1], vz + lo[2], hi[0] - lo[0] + 1, hi[1] - lo[1] + 1,
                 hi[2] - lo[2] + 1, vp, vs, rho, lo[0], lo[1], lo[2], nvy, nvz};
  // every node: Vp, Vs, density -> lambda, mu, density, and the velocity the
  // smoothing test uses (mediapar::readdata, get2in1, set_vel3d)
  const size_t n = (size_t)D.nx * D.ny * D.nz;
  std::vector<double> lam(n), mu(n), den(n), vel(n);
  for (int i = 0; i < D.nx; ++i)
    for (int j = 0; j < D.ny; ++j)
      for (int k = 0; k < D.nz; ++k) {
        const long g = D.at(i, j, k);
        double p, sv, dc;
        V.at(x[g], y[g], z[g], &p, &sv, &dc);
        const double m = dc * sv * sv;
        mu[g] = (m + m) / 2.0;
        lam[g] = ((p * p * dc - 2.0 * m) + (p * p * dc - 2.0 * m)) / 2.0;
        den[g] = (dc + dc) / 2.0;
        vel[g] = (std::fabs(p - p) < crit_value && std::fabs(p - p) / p < crit_perc)
                     ? (p + p) / 2.0
                     : (p + p) / 2.0 + 9000e3;
      }
  // cells whose velocity jumps against a neighbour: averages over sub-cell
  // samples, arithmetic for density, harmonic for lambda and mu
  // (mediapar::ApplySmooth, TwoinOne, average)
  if (sampx > 1 || sampy > 1 || sampz > 1) {
    auto over = [&](double a, double b) {
      return std::fabs(a - b) >= crit_value || std::fabs(a - b) / std::min(a, b) >= crit_perc;
    };
    const double vec3[3] = {0.0, 2.0, 4.0};
    std::vector<double> nlam(lam), nmu(mu), nden(den);
    for (int i = 3; i < ni + 3; ++i)
      for (int j = 3; j < nj + 3; ++j)
        for (int k = 3; k < nk + 3; ++k) {
          const long g = D.at(i, j, k);
          const int sx = (over(vel[g], vel[D.at(i - 1, j, k)]) || over(vel[g], vel[D.at(i + 1, j, k)])) ? sampx : 1;
          const int sy = (over(vel[g], vel[D.at(i, j - 1, k)]) || over(vel[g], vel[D.at(i, j + 1, k)])) ? sampy : 1;
          const int sz = (over(vel[g], vel[D.at(i, j, k - 1)]) || over(vel[g], vel[D.at(i, j, k + 1)])) ? sampz : 1;
          if (sx == 1 && sy == 1 && sz == 1) continue;
          double rs = 0, ms = 0, ls = 0;
          int ns = 0;
          for (int mi = 1; mi <= sx; ++mi)
            for (int mj = 1; mj <= sy; ++mj)
              for (int mk = 1; mk <= sz; ++mk) {
                const double xs = 1.0 + 2.0 / sx * (mi - 1 + 0.5);
                const double ys = 1.0 + 2.0 / sy * (mj - 1 + 0.5);
                const double zs = 1.0 + 2.0 / sz * (mk - 1 + 0.5);
                double wx[3], wy[3], wz[3], p[3] = {0, 0, 0};
                lagrange(vec3, 3, xs, wx);
                lagrange(vec3, 3, ys, wy);
                lagrange(vec3, 3, zs, wz);
                for (int a = 0; a < 3; ++a)
                  for (int b = 0; b < 3; ++b)
                    for (int c = 0; c < 3; ++c) {
                      const long q = D.at(i - 1 + a, j - 1 + b, k - 1 + c);
                      const double w = wx[a] * wy[b] * wz[c];
                      p[0] += w * x[q];
                      p[1] += w * y[q];
                      p[2] += w * z[q];
                    }
                double pv, sv, dc;
                V.at(p[0], p[1], p[2], &pv, &sv, &dc);
                const double m = dc * sv * sv, l = pv * pv * dc - 2.0 * m;
                rs += 0.5 * (dc + dc);
                // a fluid sample (mu ~ 0) resets the harmonic mu sum, as the
                // reference's TwoinOne does
                if (m < 1.e-20) ms = 0;
                else ms += 0.5 / m + 0.5 / m;
                ls += 0.5 / l + 0.5 / l;
                ++ns;
              }
          nden[g] = rs / ns;
          nmu[g] = ms > 0 ? ns * 1.0 / ms : 0.0;
          nlam[g] = ns * 1.0 / ls;
        }
    lam.swap(nlam);
    mu.swap(nmu);
    den.swap(nden);
  }
  // valid nodes to (Vp, Vs, density) (mediapar::MediaStatistics)
  std::vector<double> out[3] = {std::vector<double>(n), std::vector<double>(n),
                                std::vector<double>(n)};
  for (int i = 3; i < ni + 3; ++i)
    for (int j = 3; j < nj + 3; ++j)
      for (int k = 3; k < nk + 3; ++k) {
        const long g = D.at(i, j, k);
        out[0][g] = std::sqrt((lam[g] + 2.0 * mu[g]) / den[g]);
        out[1][g] = std::sqrt(mu[g] / den[g]);
        out[2][g] = den[g];
      }
  // ghost nodes (common::equivalence_extend): x from the nearest valid
  // node, low y and low z mirrored across the first valid node, high y and
  // high z from the last one
  for (auto &v : out) {
    for (int s = 1; s <= 3; ++s)
      for (int j = 0; j < D.ny; ++j)
        for (int k = 0; k < D.nz; ++k) {
          v[D.at(3 - s, j, k)] = v[D.at(3, j, k)];
          v[D.at(ni + 2 + s, j, k)] = v[D.at(ni + 2, j, k)];
        }
    for (int i = 0; i < D.nx; ++i)
      for (int k = 0; k < D.nz; ++k)
        for (int s = 1; s <= 3; ++s) {
          v[D.at(i, 3 - s, k)] = v[D.at(i, 3 + s, k)];
          v[D.at(i, nj + 2 + s, k)] = v[D.at(i, nj + 2, k)];
        }
    for (int i = 0; i < D.nx; ++i)
      for (int j = 0; j < D.ny; ++j)
        for (int s = 1; s <= 3; ++s) {
          v[D.at(i, j, 3 - s)] = v[D.at(i, j, 3 + s)];
          v[D.at(i, j, nk + 2 + s)] = v[D.at(i, j, nk + 2)];
        }
  }
  for (size_t g = 0; g < n; ++g) {
    alpha[g] = (float)out[0][g];
    beta[g] = (float)out[1][g];
    dens[g] = (float)out[2][g];
  }
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

}  // extern "C"

// ------------------------- point location ---------------------------------

namespace {

int locate_fail(const std::string &msg) {
  cgfd::set_global_error(("cgfd_locate_points: " + msg).c_str());
  return CGFD_ERR_ARG;
}

// Nearest node search of common::reposition over the valid nodes: squared
// distance, the first minimum in (i, j, k) order wins.  The i range is cut
// into slabs searched by threads; slab results merge in i order, so ties
// resolve as in one sequential scan.
struct Best {
  double d;
  long at;  // node index, -1: none
};

void nearest_nodes(const Dims &D, int ni, int nj, int k0, int k1, const double *x,
                   const double *y, const double *z, bool planar,
                   const std::vector<int> &pts, const double *pos, std::vector<Best> &best) {
  unsigned nth = std::thread::hardware_concurrency();
  nth = std::max(1u, std::min(nth, 16u));
  if ((long)ni * nj * (k1 - k0) * (long)pts.size() < 4000000L) nth = 1;
  nth = std::min<unsigned>(nth, (unsigned)ni);
  std::vector<std::vector<Best>> part(nth, std::vector<Best>(pts.size(), Best{1e300, -1}));
  auto work = [&](unsigned t) {
    const int i0 = 3 + (int)((long)ni * t / nth), i1 = 3 + (int)((long)ni * (t + 1) / nth);
    std::vector<Best> &b = part[t];
    for (int i = i0; i < i1; ++i)
      for (int j = 3; j < nj + 3; ++j)
        for (size_t q = 0; q < pts.size(); ++q) {
          const double *p = pos + 3 * (size_t)pts[q];
          for (int k = k0; k < k1; ++k) {
            const long c = D.at(i, j, k);
            const double dx = x[c] - p[0], dy = y[c] - p[1];
            double d = dx * dx + dy * dy;
            if (!planar) {
              const double dz = z[c] - p[2];
              d += dz * dz;
            }
            if (d < b[q].d) b[q] = Best{d, c};
          }
        }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nth; ++t) th.emplace_back(work, t);
  work(0);
  for (auto &t : th) t.join();
  for (size_t q = 0; q < pts.size(); ++q) {
    Best b{1e300, -1};
    for (unsigned t = 0; t < nth; ++t)
      if (part[t][q].d < b.d) b = part[t][q];
    best[q] = b;
  }
}

// The Gaussian weights of cal_norm (src/source.cpp:345-378): a 7^3 block of
// exp(-(s/1.5)^2)/(sqrt(pi) 1.5) products, s the node offset minus the
// sub-cell shift, normalised to sum 1; when the block reaches above the
// surface (iz + 3 > top) it is normalised again over its nodes at or below
// the surface (iz is the node the search found, before any shift).
bool norm_block(double shx, double shy, double shz, int iz, int top, double *w) {
  const double a = 1.5;
  auto g = [&](double s) { return std::exp(-s * s / (a * a)) / (std::sqrt(kPi) * a); };
  double sum = 0.0;
  for (int i = -3; i <= 3; ++i)
    for (int j = -3; j <= 3; ++j)
      for (int k = -3; k <= 3; ++k) {
        const double v = g(i - shx) * g(j - shy) * g(k - shz);
        w[((i + 3) * 7 + (j + 3)) * 7 + (k + 3)] = v;
        sum += v;
      }
  if (sum < 1e-20) return false;
  for (int q = 0; q < 343; ++q) w[q] /= sum;
  if (iz + 3 > top) {
    sum = 0.0;
    const int kn = top + 1 - iz + 3;  // block layers at or below the surface
    for (int i = 0; i < 7; ++i)
      for (int j = 0; j < 7; ++j)
        for (int k = 0; k < kn; ++k) sum += w[(i * 7 + j) * 7 + k];
    for (int q = 0; q < 343; ++q) w[q] /= sum;
  }
  return true;
}

// Force points (eighth_locate, src/source.cpp:277-343, applied four times):
// the 3^3 nodes around the point are refined to 5^3 by Lagrange
// interpolation in index space (nodes at 0, 2, 4); the nearest of the 125
// gives the step s in {-2..2} of this level and the centre of the next
// level's 3^3 block.  The shift is sum s_l / 2^(l+1).
bool force_shift(const Dims &D, const double *x, const double *y, const double *z,
                 const int *loc, const double *p, double sh[3]) {
  double m[3][27];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) {
        const long g = D.at(loc[0] - 1 + a, loc[1] - 1 + b, loc[2] - 1 + c);
        m[0][(a * 3 + b) * 3 + c] = x[g];
        m[1][(a * 3 + b) * 3 + c] = y[g];
        m[2][(a * 3 + b) * 3 + c] = z[g];
      }
  const double nodes[3] = {0.0, 2.0, 4.0};
  double W[5][3];  // Lagrange weights at 0..4 of the nodes 0, 2, 4
  for (int t = 0; t < 5; ++t) lagrange(nodes, 3, (double)t, W[t]);
  sh[0] = sh[1] = sh[2] = 0.0;
  for (int lev = 0; lev < 4; ++lev) {
    double f[3][125];
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        for (int k = 0; k < 5; ++k) {
          const int o = (i * 5 + j) * 5 + k;
          if (i % 2 == 0 && j % 2 == 0 && k % 2 == 0) {
            for (int q = 0; q < 3; ++q) f[q][o] = m[q][((i / 2) * 3 + j / 2) * 3 + k / 2];
            continue;
          }
          for (int q = 0; q < 3; ++q) {
            double v = 0.0;
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) v += W[i][a] * W[j][b] * W[k][c] * m[q][(a * 3 + b) * 3 + c];
            f[q][o] = v;
          }
        }
    double best = 1e20;
    int bi = -1, bj = -1, bk = -1;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        for (int k = 0; k < 5; ++k) {
          const int o = (i * 5 + j) * 5 + k;
          const double dx = f[0][o] - p[0], dy = f[1][o] - p[1], dz = f[2][o] - p[2];
          const double d = dx * dx + dy * dy + dz * dz;
          if (d < best) { best = d; bi = i; bj = j; bk = k; }
        }
    // the next level's block must lie inside the 5^3 one
    if (bi < 1 || bi > 3 || bj < 1 || bj > 3 || bk < 1 || bk > 3) return false;
    const double s = 1.0 / (double)(2 << lev);
    sh[0] += (bi - 2) * s;
    sh[1] += (bj - 2) * s;
    sh[2] += (bk - 2) * s;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c)
          for (int q = 0; q < 3; ++q)
            m[q][(a * 3 + b) * 3 + c] = f[q][((bi + a - 1) * 5 + bj + b - 1) * 5 + bk + c - 1];
  }
  return true;
}

// Moment and focal points (MomentShiftPosition, src/source.cpp:157-275): the
// cells within one node in x and y and three in z of the point's node are
// sampled trilinearly at 1/8 of the index spacing; the nearest sample moves
// the point's node to the nearest whole index and leaves a shift in
// [-1/2, 3/8] per axis.
bool moment_shift(const Dims &D, const double *x, const double *y, const double *z, int *loc,
                  const double *p, double sh[3]) {
  const int ns = 8;
  double best = 1e20;
  int b[3] = {-1, -1, -1};
  const double *v[3] = {x, y, z};
  for (int si = -1; si <= 0; ++si)
    for (int sj = -1; sj <= 0; ++sj)
      for (int sk = -3; sk <= 2; ++sk) {
        double c[3][8];
        for (int a = 0; a < 2; ++a)
          for (int bb = 0; bb < 2; ++bb)
            for (int cc = 0; cc < 2; ++cc) {
              const long g = D.at(loc[0] + si + a, loc[1] + sj + bb, loc[2] + sk + cc);
              for (int q = 0; q < 3; ++q) c[q][(a * 2 + bb) * 2 + cc] = v[q][g];
            }
        for (int mi = 0; mi < ns; ++mi)
          for (int mj = 0; mj < ns; ++mj)
            for (int mk = 0; mk < ns; ++mk) {
              const double nodes[2] = {0.0, 1.0};
              double wx[2], wy[2], wz[2];
              lagrange(nodes, 2, (double)mi / ns, wx);
              lagrange(nodes, 2, (double)mj / ns, wy);
              lagrange(nodes, 2, (double)mk / ns, wz);
              double d = 0.0;
              for (int q = 0; q < 3; ++q) {
                double f = 0.0;
                for (int a = 0; a < 2; ++a)
                  for (int bb = 0; bb < 2; ++bb)
                    for (int cc = 0; cc < 2; ++cc) f += wx[a] * wy[bb] * wz[cc] * c[q][(a * 2 + bb) * 2 + cc];
                d += (f - p[q]) * (f - p[q]);
              }
              // the samples are ordered by their position in the 16 x 16 x 48
              // sub-grid (i, then j, then k), as the reference scans them
              const int gi = (si + 1) * ns + mi, gj = (sj + 1) * ns + mj, gk = (sk + 3) * ns + mk;
              if (d < best ||
                  (d == best && (gi < b[0] || (gi == b[0] && (gj < b[1] || (gj == b[1] && gk < b[2])))))) {
                best = d;
                b[0] = gi; b[1] = gj; b[2] = gk;
              }
            }
      }
  if (b[0] < 0) return false;
  const int half[3] = {1, 1, 3};
  for (int q = 0; q < 3; ++q) {
    const int s = (b[q] + ns / 2) / ns;
    loc[q] += s - half[q];
    sh[q] = (double)(b[q] - s * ns) / ns;
  }
  return true;
}

}  // namespace

extern "C" {

int cgfd_locate_points(int ni, int nj, int nk, const double *x, const double *y, const double *z,
                       double hyper_height, int n, const double *pos, int *loc, double *posz) {
  CGFD_ABI_BEGIN
  if (ni < 1 || nj < 1 || nk < 1 || n < 0 || (n > 0 && (!x || !y || !z || !pos || !loc)))
    return locate_fail("bad arguments");
  const Dims D{ni + 6, nj + 6, nk + 6};
  const int top = nk + 2;
  std::vector<int> above, below;
  for (int q = 0; q < n; ++q) (pos[3 * q + 2] > hyper_height ? above : below).push_back(q);
  std::vector<Best> ba(above.size()), bb(below.size());
  if (!above.empty()) nearest_nodes(D, ni, nj, top, top + 1, x, y, z, true, above, pos, ba);
  if (!below.empty()) nearest_nodes(D, ni, nj, 3, nk + 3, x, y, z, false, below, pos, bb);
  auto put = [&](const std::vector<int> &pts, const std::vector<Best> &best, bool surf) {
    for (size_t t = 0; t < pts.size(); ++t) {
      const int q = pts[t];
      if (best[t].at < 0) return false;
      const long c = best[t].at;
      loc[3 * q] = (int)(c / ((long)D.ny * D.nz));
      loc[3 * q + 1] = (int)(c / D.nz % D.ny);
      loc[3 * q + 2] = (int)(c % D.nz);
      if (posz) posz[q] = surf ? z[c] : pos[3 * q + 2];
    }
    return true;
  };
  if (!put(above, ba, true) || !put(below, bb, false))
    return locate_fail("no finite distance to any valid node");
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

int cgfd_source_smoothing(int ni, int nj, int nk, const double *x, const double *y,
                          const double *z, int kind, int n, const double *pos, int *loc,
                          double *weights) {
  CGFD_ABI_BEGIN
  if (ni < 1 || nj < 1 || nk < 1 || n < 0 || (kind != 0 && kind != 1) ||
      (n > 0 && (!x || !y || !z || !pos || !loc || !weights)))
    return locate_fail("bad smoothing arguments");
  const Dims D{ni + 6, nj + 6, nk + 6};
  const int top = nk + 2;
  for (int q = 0; q < n; ++q) {
    int *l = loc + 3 * q;
    if (l[0] < 3 || l[0] >= ni + 3 || l[1] < 3 || l[1] >= nj + 3 || l[2] < 3 || l[2] > top)
      return locate_fail("source outside the valid grid");
    const int iz = l[2];
    double sh[3];
    const bool ok = kind == 0 ? force_shift(D, x, y, z, l, pos + 3 * q, sh)
                              : moment_shift(D, x, y, z, l, pos + 3 * q, sh);
    if (!ok) return locate_fail("sub-cell search left its block");
    if (l[0] < 3 || l[0] >= ni + 3 || l[1] < 3 || l[1] >= nj + 3 || l[2] < 3 || l[2] > top)
      return locate_fail("shifted source outside the valid grid");
    if (!norm_block(sh[0], sh[1], sh[2], iz, top, weights + (size_t)343 * q))
      return locate_fail("smoothing weights sum to zero");
  }
  return CGFD_OK;
  CGFD_ABI_END(nullptr)
}

}  // extern "C"
