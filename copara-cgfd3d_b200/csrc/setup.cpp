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
#include "../../include/cgfd.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
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

int grid_fail(const std::string &msg) {
  cgfd::set_global_error(("cgfd_grid_vmap: " + msg).c_str());
  return CGFD_ERR_ARG;
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

int cgfd_grid_vmap(int ni, int nj, int nk, int nsurf, const int *gridpoints,
                   const int *equalspacing, const double *anchor, int hybrid,
                   double convers_depth, double *x, double *y, double *z, int *con_index) {
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
    for (int j = 0; j < nj; ++j)
      for (int q = 1; q < nsurf; ++q)
        if (col(i, j)[2 + q] > col(i, j)[1 + q])
          return grid_fail("interface depths must decrease from the top down");

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
      gp[l] = (int)(nk * (hi[l] - lo[l]) / total_len);
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
}

}  // extern "C"
