// wavesim.cpp -- wavesim_b200: the B200 solver driven by the reference's own
// input files, through the C ABI of libcgfd.so only.
//
//   wavesim_b200 SeisFD3D.conf [--device N] [--steps N] [--out DIR]
//                              [--storage f32|f16|bf16] [--dump FILE]
//
// It replaces the reference's wavesim (src/simulation.cc) for one GPU: the
// same par file (SeisFD3D.conf) and the files it names -- the vmap grid, the
// volume media (NetCDF classic), absorb.dat, source.dat (point forces and
// moments, or a finite-fault series file in NetCDF classic) and station.dat
// (receivers, receiver lines, snapshots) -- are read with the reference's
// column semantics (common::get_conf: the value is the numcol-th
// whitespace-separated token of the first line, not starting with '#',
// whose first token is the key; src/common.cpp:23-59, 280-333), and the
// outputs are the reference's seismo.nc, peakvel.nc and snap_NNN.nc
// variables, in NetCDF classic.  --dump writes the pre-processed model
// (grid metric, media, PML, sources, receivers) as a flat binary instead of
// running the solver (tests compare it with the reference's own host code).
#include "../../include/cgfd.h"
#include "../csrc/ncwrite.h"

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

constexpr int LFD = 3;

[[noreturn]] void die(const std::string &msg) {
  std::fprintf(stderr, "wavesim_b200: %s\n", msg.c_str());
  std::exit(1);
}

void check(int st, const char *what, cgfd_solver *h = nullptr) {
  if (st == CGFD_OK) return;
  char buf[1024];
  cgfd_last_error(h, buf, sizeof(buf));
  die(std::string(what) + " failed (" + std::to_string(st) + "): " + buf);
}

// A par file: common::get_conf's lookup, and the token stream after an
// anchor line (common::setchunk followed by fscanf).
struct Par {
  std::string path;
  std::vector<std::string> lines;
  explicit Par(const std::string &p) : path(p) {
    std::ifstream f(p);
    if (!f) die("cannot open " + p);
    for (std::string l; std::getline(f, l);) lines.push_back(l);
  }
  static std::vector<std::string> tokens(const std::string &l) {
    std::istringstream s(l);
    std::vector<std::string> t;
    for (std::string w; s >> w;) t.push_back(w);
    return t;
  }
  bool has(const std::string &key, int col = 3) const {
    std::string v;
    return find(key, col, &v);
  }
  bool find(const std::string &key, int col, std::string *out) const {
    for (const std::string &l : lines) {
      if (!l.empty() && l[0] == '#') continue;
      const std::vector<std::string> t = tokens(l);
      if (!t.empty() && t[0] == key && (int)t.size() >= col) {
        *out = t[col - 1];
        return true;
      }
    }
    return false;
  }
  std::string str(const std::string &key, int col = 3) const {
    std::string v;
    if (!find(key, col, &v))
      die("no value at column " + std::to_string(col) + " for " + key + " in " + path);
    return v;
  }
  // an integer (atoi's reading: leading digits, 0 for none), refused beyond
  // half the int range so that index arithmetic on it cannot overflow
  int i(const std::string &key, int col = 3) const {
    const long long v = std::strtoll(str(key, col).c_str(), nullptr, 10);
    if (v > INT_MAX / 2 || v < INT_MIN / 2)
      die(key + " in " + path + ": integer out of range");
    return (int)v;
  }
  double d(const std::string &key, int col = 3) const { return std::atof(str(key, col).c_str()); }
  // whitespace tokens after the line whose first token is `anchor`
  std::vector<std::string> after(const std::string &anchor) const {
    std::vector<std::string> out;
    bool on = false;
    for (const std::string &l : lines) {
      if (!on) {
        if (!l.empty() && l[0] == '#') continue;
        const std::vector<std::string> t = tokens(l);
        if (!t.empty() && t[0] == anchor) on = true;
        continue;
      }
      for (const std::string &w : tokens(l)) out.push_back(w);
    }
    if (!on) die("no anchor " + anchor + " in " + path);
    return out;
  }
};

std::string join(const std::string &dir, const std::string &name) {
  if (name.empty() || name[0] == '/') return name;
  return dir + "/" + name;
}

struct Point {
  double x, y, z;
  int pnum, lnum;
};

struct Snap {
  int s[3], n[3], d[3], tinv, cmp;
};

// bounds on what a par file may ask for, far above any model that fits a GPU:
// cells along one axis, time steps, receivers and sources of one kind
constexpr int kMaxCells = 1 << 20, kMaxSteps = 1 << 28, kMaxPoints = 1 << 24;

struct Model {
  int ni, nj, nk, nt, con = 0, nabs[6] = {0, 0, 0, 0, 0, 0};
  double steph, stept;
  size_t N = 0;
  std::vector<double> x, y, z, metric[10];
  std::vector<float> alpha, beta, rho;
  std::vector<double> pml[9];
  // sources
  std::vector<int> mloc, floc, focloc;
  std::vector<float> m6, f3, mstf, fstf, focmom;
  int nfoc = 0, fnt = 0;
  double fdt = 0.0;
  // receivers and snapshots
  std::vector<Point> recv;
  std::vector<int> rloc;
  std::vector<float> rpos;  // the receivers' positions, z as located
  int seis_tinv = 1;
  std::vector<Snap> snaps;
  bool peakvel = false;
};

// the vmap grid (gridmesh::read_vmapnew, src/gridmesh.cpp:72-130)
void read_grid(const Par &conf, const std::string &dir, Model &m) {
  const std::string type = conf.str("grid_type");
  if (type != "vmap") die("grid_type " + type + ": only vmap grids are read");
  const Par g(join(dir, conf.str("grid_filename")));
  const int hybrid = conf.i("hybrid_grid");
  const double convers = conf.d("conversion_interface_depth");
  const int d0 = g.i("vmap_dims", 3), d1 = g.i("vmap_dims", 4), nsurf = g.i("vmap_dims", 5);
  if (d0 != m.ni || d1 != m.nj) die("vmap_dims differ from ni, nj");
  if (nsurf < 2) die("vmap_dims: at least 2 interfaces");
  std::vector<int> gp(nsurf - 1), eq(nsurf - 1);
  for (int l = 0; l < nsurf - 1; ++l) {
    gp[l] = g.i("vmap_gridpoints", 3 + l);
    eq[l] = g.str("vmap_equalspacing", 3 + l) == "0" ? 0 : 1;
  }
  const std::vector<std::string> t = g.after("<vmap_anchor>");
  const size_t need = (size_t)m.ni * m.nj * (2 + nsurf);
  if (t.size() < need) die("vmap anchor block too short");
  std::vector<double> anchor(need);
  for (size_t q = 0; q < need; ++q) anchor[q] = std::atof(t[q].c_str());
  m.x.assign(m.N, 0.0);
  m.y.assign(m.N, 0.0);
  m.z.assign(m.N, 0.0);
  check(cgfd_grid_vmap(m.ni, m.nj, m.nk, nsurf, gp.data(), eq.data(), anchor.data(), hybrid,
                       convers, m.x.data(), m.y.data(), m.z.data(), &m.con),
        "cgfd_grid_vmap");
  if (!hybrid) die("hybrid_grid must be 1 (the solver's SimpleCar path)");
  double *out[10];
  for (int q = 0; q < 10; ++q) {
    m.metric[q].assign(m.N, 0.0);
    out[q] = m.metric[q].data();
  }
  check(cgfd_metric_from_coords(m.ni, m.nj, m.nk, m.steph, m.x.data(), m.y.data(), m.z.data(),
                                out),
        "cgfd_metric_from_coords");
}

// volume media from its NetCDF classic file (mediapar, src/mediaparas.cpp)
void read_media(const Par &conf, const std::string &dir, Model &m) {
  const std::string type = conf.str("media_type");
  if (type != "volume") die("media_type " + type + ": only volume media are read");
  const std::string path = join(dir, conf.str("media_filename"));
  int n[3] = {0, 0, 0};
  check(cgfd_read_media_volume_nc(path.c_str(), &n[0], &n[1], &n[2], nullptr, nullptr, nullptr,
                                  nullptr, nullptr, nullptr),
        "cgfd_read_media_volume_nc");
  std::vector<double> vx(n[0]), vy(n[1]), vz(n[2]);
  const size_t nv = (size_t)n[0] * n[1] * n[2];
  std::vector<float> vp(nv), vs(nv), rho(nv);
  check(cgfd_read_media_volume_nc(path.c_str(), &n[0], &n[1], &n[2], vx.data(), vy.data(),
                                  vz.data(), vp.data(), vs.data(), rho.data()),
        "cgfd_read_media_volume_nc");
  m.alpha.assign(m.N, 0.f);
  m.beta.assign(m.N, 0.f);
  m.rho.assign(m.N, 0.f);
  // sub-cell samples per axis where the velocity jumps (ApplySmooth takes
  // the par value as the count; 0 and 1 both mean none)
  int samp[3];
  for (int a = 0; a < 3; ++a) {
    samp[a] = conf.i("sampling_point_per_cell", 3 + a);
    if (samp[a] < 1) samp[a] = 1;
  }
  check(cgfd_media_volume(m.ni, m.nj, m.nk, m.x.data(), m.y.data(), m.z.data(), n[0], n[1],
                          n[2], vx.data(), vy.data(), vz.data(), vp.data(), vs.data(),
                          rho.data(), conf.d("threshold_velocity_jump_of_interface"),
                          conf.d("threshold_percent_change_of_interface"), samp[0], samp[1],
                          samp[2], m.alpha.data(), m.beta.data(), m.rho.data()),
        "cgfd_media_volume");
}

// absorb.dat and CalCFSfactors (src/absorb.cpp:26-44, 346-805): the layer
// thicknesses follow the metric along the first valid row of each axis
void read_absorb(const Par &conf, const std::string &dir, Model &m) {
  const Par a(join(dir, conf.str("absorb_filename")));
  double vel[6], bmax[6], amax[6];
  for (int q = 0; q < 6; ++q) {
    m.nabs[q] = a.i("abs_number", 3 + q);
    vel[q] = a.d("abs_velocity", 3 + q);
    bmax[q] = a.d("bmax", 3 + q);
    amax[q] = a.d("amax", 3 + q);
  }
  if (m.nabs[5] != 0) die("abs_number: the top (Z2) must be 0 (free surface)");
  const int nx = m.ni + 6, ny = m.nj + 6, nz = m.nk + 6;
  auto g = [&](int i, int j, int k) { return ((size_t)i * ny + j) * nz + k; };
  auto dl = [&](int q0, size_t p) {
    const double a0 = m.metric[q0][p], a1 = m.metric[q0 + 1][p], a2 = m.metric[q0 + 2][p];
    const double n = std::sqrt(a0 * a0 + a1 * a1 + a2 * a2);
    return n > 0 ? m.steph / n : 0.0;
  };
  std::vector<double> dlx(nx), dly(ny), dlz(nz);
  for (int i = 0; i < nx; ++i) dlx[i] = dl(0, g(i, LFD, LFD));
  for (int j = 0; j < ny; ++j) dly[j] = dl(3, g(LFD, j, LFD));
  for (int k = 0; k < nz; ++k) dlz[k] = dl(6, g(LFD, LFD, k));
  const int n3[3] = {nx, ny, nz};
  for (int q = 0; q < 9; ++q) m.pml[q].assign(n3[q % 3], 0.0);
  check(cgfd_cfs_factors(m.ni, m.nj, m.nk, m.nabs, vel, bmax, amax, dlx.data(), dly.data(),
                         dlz.data(), m.pml[0].data(), m.pml[1].data(), m.pml[2].data(),
                         m.pml[3].data(), m.pml[4].data(), m.pml[5].data(), m.pml[6].data(),
                         m.pml[7].data(), m.pml[8].data()),
        "cgfd_cfs_factors");
}

void locate(const Model &m, double hyper, std::vector<double> &pos, std::vector<int> &loc,
            const char *what) {
  const int n = (int)(pos.size() / 3);
  loc.assign(3 * n, 0);
  std::vector<double> posz(n);
  check(cgfd_locate_points(m.ni, m.nj, m.nk, m.x.data(), m.y.data(), m.z.data(), hyper, n,
                           pos.data(), loc.data(), posz.data()),
        what);
  for (int q = 0; q < n; ++q) pos[3 * q + 2] = posz[q];
}

int stf_type(const std::string &name) {
  static const char *names[8] = {"Gauss", "gauss", "Ricker", "ricker",
                                 "Bell", "bell", "BELL", "Step"};
  for (int q = 0; q < 8; ++q)
    if (name == names[q]) return q;
  die("unknown source time function " + name);
}

// source.dat (source::source, readdata, cal_index; src/source.cpp:23-70,
// 686-840, 1040-1160)
void read_sources(const Par &conf, const std::string &dir, Model &m) {
  const Par s(join(dir, conf.str("source_filename")));
  const double d2m = s.d("distance2meter");
  const double hyper = s.d("source_hyper_height") * d2m;
  const int type = s.i("source_type");
  const int nstf = 2 * (m.nt + 1);
  if (type == 1) {  // finite fault from its NetCDF classic file
    const std::string path = join(dir, s.str("focal_process_NC_file"));
    int np = 0, fnt = 0;
    double fdt = 0;
    check(cgfd_read_focal_nc(path.c_str(), &np, &fnt, &fdt, nullptr, nullptr, nullptr, nullptr),
          "cgfd_read_focal_nc");
    std::vector<double> px(np), py(np), pz(np);
    m.focmom.assign((size_t)6 * np * fnt, 0.f);
    check(cgfd_read_focal_nc(path.c_str(), &np, &fnt, &fdt, px.data(), py.data(), pz.data(),
                             m.focmom.data()),
          "cgfd_read_focal_nc");
    const double damp = s.has("simulate_damp") ? s.d("simulate_damp") : 1.0;
    for (float &v : m.focmom) v = (float)(v * damp);
    std::vector<double> pos(3 * np);
    for (int q = 0; q < np; ++q) {
      pos[3 * q] = px[q];
      pos[3 * q + 1] = py[q];
      pos[3 * q + 2] = pz[q];
    }
    locate(m, hyper, pos, m.focloc, "locating the focal points");
    m.nfoc = np;
    m.fnt = fnt;
    m.fdt = fdt;
    return;
  }
  if (type != 2 && type != 3) die("source_type must be 1, 2 or 3");
  const int nfrc = s.i("number_of_force_source"), nmnt = s.i("number_of_moment_source");
  if (nfrc < 0 || nmnt < 0 || nfrc > kMaxPoints || nmnt > kMaxPoints)
    die("number_of_force_source or number_of_moment_source out of range");
  std::vector<double> stf(nstf);
  if (nfrc > 0) {
    const int nwin = s.i("force_stf_window");
    const std::vector<std::string> t = s.after("<anchor_force>");
    if (t.size() / 8 < (size_t)nfrc) die("force block too short");
    std::vector<double> pos(3 * nfrc), start(nfrc);
    m.f3.assign(3 * nfrc, 0.f);
    for (int q = 0; q < nfrc; ++q) {
      const double *v = nullptr;
      double r[8];
      for (int c = 0; c < 8; ++c) r[c] = std::atof(t[8 * q + c].c_str());
      v = r;
      for (int c = 0; c < 3; ++c) pos[3 * q + c] = v[c] * d2m;
      start[q] = v[3];
      for (int c = 0; c < 3; ++c) m.f3[3 * q + c] = (float)(v[5 + c] * v[4]);
    }
    locate(m, hyper, pos, m.floc, "locating the forces");
    m.fstf.assign((size_t)nfrc * nstf, 0.f);
    // each window overwrites the series (the reference keeps the last)
    for (int q = 0; q < nfrc; ++q)
      for (int w = 0; w < nwin; ++w)
        check(cgfd_stf(stf_type(s.str("force_stf_type", 3 + w)), start[q],
                       s.d("force_stf_timefactor", 3 + w), s.d("force_stf_freqfactor", 3 + w),
                       nstf, m.stept / 2.0, m.fstf.data() + (size_t)q * nstf),
              "cgfd_stf");
  }
  if (nmnt > 0) {
    const int nwin = s.i("moment_stf_window");
    const std::string mech = s.str("moment_mech_input");
    if (mech != "moment" && mech != "angle") die("moment_mech_input must be moment or angle");
    const int ncol = mech == "moment" ? 11 : 8;
    const std::vector<std::string> t = s.after("<anchor_moment>");
    if (t.size() / ncol < (size_t)nmnt) die("moment block too short");
    std::vector<double> pos(3 * nmnt), start(nmnt);
    m.m6.assign(6 * nmnt, 0.f);
    for (int q = 0; q < nmnt; ++q) {
      double r[11];
      for (int c = 0; c < ncol; ++c) r[c] = std::atof(t[ncol * q + c].c_str());
      for (int c = 0; c < 3; ++c) pos[3 * q + c] = r[c] * d2m;
      start[q] = r[3];
      double mm[6];
      if (mech == "moment") {
        for (int c = 0; c < 6; ++c) mm[c] = r[5 + c];
      } else {
        check(cgfd_angle2moment(r[5], r[6], r[7], mm), "cgfd_angle2moment");
      }
      for (int c = 0; c < 6; ++c) m.m6[6 * q + c] = (float)(mm[c] * r[4]);
    }
    locate(m, hyper, pos, m.mloc, "locating the moments");
    if (mech == "angle")  // x mu at the source node (src/source.cpp:1127-1135)
      for (int q = 0; q < nmnt; ++q) {
        const size_t g = ((size_t)m.mloc[3 * q] * (m.nj + 6) + m.mloc[3 * q + 1]) * (m.nk + 6) +
                         m.mloc[3 * q + 2];
        const float mu = m.rho[g] * m.beta[g] * m.beta[g];
        for (int c = 0; c < 6; ++c) m.m6[6 * q + c] *= mu;
      }
    m.mstf.assign((size_t)nmnt * nstf, 0.f);
    for (int q = 0; q < nmnt; ++q)
      for (int w = 0; w < nwin; ++w)
        check(cgfd_stf(stf_type(s.str("moment_stf_type", 3 + w)), start[q],
                       s.d("moment_stf_timefactor", 3 + w), s.d("moment_stf_freqfactor", 3 + w),
                       nstf, m.stept / 2.0, m.mstf.data() + (size_t)q * nstf),
              "cgfd_stf");
  }
}

// station.dat (seisplot::seisplot + readdata + locpoint; src/seisplot.cpp:
// 23-60, 336-440)
void read_stations(const Par &conf, const std::string &dir, Model &m) {
  const Par s(join(dir, conf.str("station_filename")));
  m.peakvel = conf.has("output_peakvel") && conf.i("output_peakvel") != 0;
  const double hyper = s.d("topo_hyper_height");
  m.seis_tinv = s.i("tinv_of_seismo");
  if (m.seis_tinv < 1) die("tinv_of_seismo must be at least 1");
  const int nsnap = s.i("number_of_snap"), nline = s.i("number_of_inline");
  const int nrecv = s.i("number_of_recv");
  if (nsnap < 0 || nline < 0 || nrecv < 0 || nsnap > 999 || nline > 999 || nrecv > kMaxPoints)
    die("number_of_snap, number_of_inline or number_of_recv out of range");
  const int last[3] = {m.ni + LFD - 1, m.nj + LFD - 1, m.nk + LFD - 1};
  char key[32];
  for (int q = 0; q < nsnap; ++q) {
    std::snprintf(key, sizeof(key), "snap_%3.3d", q + 1);
    Snap sn;
    for (int a = 0; a < 3; ++a) {
      sn.s[a] = s.i(key, 3 + a) - 1 + LFD;  // 1-based valid index -> full array
      sn.n[a] = s.i(key, 6 + a);
      sn.d[a] = s.i(key, 9 + a);
    }
    sn.tinv = s.i(key, 12);
    sn.cmp = s.i(key, 13);
    if (sn.tinv < 1 || sn.cmp < 1 || sn.cmp > 3) die(std::string(key) + ": bad tinv or cmp");
    for (int a = 0; a < 3; ++a)
      if (sn.s[a] < LFD || sn.n[a] < 1 || sn.d[a] < 1 ||
          sn.s[a] + (long long)(sn.n[a] - 1) * sn.d[a] > last[a])
        die(std::string(key) + ": start, count and stride must stay inside the grid");
    m.snaps.push_back(sn);
  }
  for (int q = 0; q < nrecv; ++q) {
    std::snprintf(key, sizeof(key), "recv_%3.3d", q + 1);
    m.recv.push_back({s.d(key, 3), s.d(key, 4), s.d(key, 5), q, 0});
  }
  for (int l = 0; l < nline; ++l) {
    std::snprintf(key, sizeof(key), "line_%3.3d", l + 1);
    const double x0 = s.d(key, 3), y0 = s.d(key, 4), z0 = s.d(key, 5);
    const double dx = s.d(key, 7), dy = s.d(key, 8), dz = s.d(key, 9);
    const double fnum = s.d(key, 11);
    if (!(fnum >= 0 && fnum <= kMaxPoints)) die(std::string(key) + ": receiver count out of range");
    const int num = (int)fnum;
    if (m.recv.size() + (size_t)num > (size_t)kMaxPoints) die("too many receivers");
    for (int j = 0; j < num; ++j) m.recv.push_back({x0 + j * dx, y0 + j * dy, z0 + j * dz, j, l + 1});
  }
  std::vector<double> pos(3 * m.recv.size());
  for (size_t q = 0; q < m.recv.size(); ++q) {
    pos[3 * q] = m.recv[q].x;
    pos[3 * q + 1] = m.recv[q].y;
    pos[3 * q + 2] = m.recv[q].z;
  }
  if (!m.recv.empty()) locate(m, hyper, pos, m.rloc, "locating the receivers");
  m.rpos.assign(pos.begin(), pos.end());
}

void write_seismo(const std::string &path, const Model &m, const std::vector<float> &seis,
                  int done) {
  const int n = (int)m.recv.size(), tinv = m.seis_tinv;
  const int nrec = (done + tinv - 1) / tinv;  // steps t with t % tinv == 0
  std::vector<std::vector<float>> comp(9, std::vector<float>((size_t)nrec * n));
  for (int c = 0; c < 9; ++c)
    for (int r = 0; r < n; ++r)
      for (int q = 0; q < nrec; ++q)
        comp[c][(size_t)q * n + r] = seis[((size_t)c * n + r) * m.nt + (size_t)q * tinv];
  std::vector<float> tcur(nrec), px(n), py(n), pz(n);
  std::vector<int> pnum(n), lnum(n);
  for (int q = 0; q < nrec; ++q) tcur[q] = (float)((q * tinv + 1) * m.stept);
  for (int r = 0; r < n; ++r) {
    pnum[r] = m.recv[r].pnum;
    lnum[r] = m.recv[r].lnum;
    px[r] = m.rpos[3 * r];
    py[r] = m.rpos[3 * r + 1];
    pz[r] = m.rpos[3 * r + 2];
  }
  using namespace cgfd::nc;
  static const char *names[9] = {"Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Txy", "Txz", "Tyz"};
  std::vector<Dim> dims = {{"TimeNum", 0}, {"PointNum", (size_t)n}};
  std::vector<Var> vars;
  for (int c = 0; c < 9; ++c) vars.push_back({names[c], NC_FLOAT, {0, 1}, comp[c].data()});
  vars.push_back({"currTime", NC_FLOAT, {0}, tcur.data()});
  vars.push_back({"Pnum", NC_INT, {1}, pnum.data()});
  vars.push_back({"Lnum", NC_INT, {1}, lnum.data()});
  vars.push_back({"posx", NC_FLOAT, {1}, px.data()});
  vars.push_back({"posy", NC_FLOAT, {1}, py.data()});
  vars.push_back({"posz", NC_FLOAT, {1}, pz.data()});
  const std::string content("Velocity and Stress seismogram", 31);
  if (!write_classic(path.c_str(), dims, {{"Content", content}}, vars, (size_t)nrec))
    die("cannot write " + path);
}

// one snapshot file per snap_NNN: the sub-volume of V (cmp 1), T (cmp 2) or
// both (cmp 3) every tinv steps, [time][i][j][k] per component
struct SnapWriter {
  std::string path;
  const Snap *sn;
  std::vector<std::vector<float>> data;  // per component, all times
  int ntime = 0;
  unsigned mask() const { return sn->cmp == 1 ? 0x7u : sn->cmp == 2 ? 0x1f8u : 0x1ffu; }
  void take(cgfd_solver *h) {
    const size_t cells = (size_t)sn->n[0] * sn->n[1] * sn->n[2];
    const unsigned mk = mask();
    const int nc = __builtin_popcount(mk);
    std::vector<float> buf(cells * nc);
    check(cgfd_get_snapshot(h, CGFD_SET_FW, sn->s, sn->n, sn->d, (int)mk, buf.data()),
          "cgfd_get_snapshot", h);
    if (data.empty()) data.resize(nc);
    for (int c = 0; c < nc; ++c)
      data[c].insert(data[c].end(), buf.begin() + c * cells, buf.begin() + (c + 1) * cells);
    ++ntime;
  }
  void write(double stept) const {
    using namespace cgfd::nc;
    static const char *names[9] = {"Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Txy", "Txz", "Tyz"};
    std::vector<Dim> dims = {{"time", 0}, {"I", (size_t)sn->n[0]}, {"J", (size_t)sn->n[1]},
                             {"K", (size_t)sn->n[2]}};
    std::vector<Var> vars;
    const unsigned mk = mask();
    int q = 0;
    for (int c = 0; c < 9; ++c)
      if (mk & (1u << c)) vars.push_back({names[c], NC_FLOAT, {0, 1, 2, 3}, data[q++].data()});
    std::vector<float> t(ntime);
    for (int k = 0; k < ntime; ++k) t[k] = (float)((k * sn->tinv + 1) * stept);
    vars.push_back({"time", NC_FLOAT, {0}, t.data()});
    if (!write_classic(path.c_str(), dims, {{"Content", std::string("wave field snapshot")}},
                       vars, (size_t)ntime))
      die("cannot write " + path);
  }
};

template <class T>
void dump_vec(FILE *f, const std::vector<T> &v) {
  const long long n = (long long)v.size();
  std::fwrite(&n, sizeof(n), 1, f);
  if (n) std::fwrite(v.data(), sizeof(T), v.size(), f);
}

// the pre-processed model, for tests: header ints, then each array with its
// length
void dump(const std::string &path, const Model &m) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) die("cannot write " + path);
  const int hdr[12] = {m.ni, m.nj, m.nk, m.nt, m.con, m.nabs[0], m.nabs[1], m.nabs[2],
                       m.nabs[3], m.nabs[4], m.nabs[5], m.nfoc};
  std::fwrite(hdr, sizeof(int), 12, f);
  const double dd[3] = {m.steph, m.stept, m.fdt};
  std::fwrite(dd, sizeof(double), 3, f);
  dump_vec(f, m.x);
  dump_vec(f, m.y);
  dump_vec(f, m.z);
  for (int q : {6, 7, 8, 9}) dump_vec(f, m.metric[q]);  // zeta_x zeta_y zeta_z jac
  dump_vec(f, m.alpha);
  dump_vec(f, m.beta);
  dump_vec(f, m.rho);
  for (int q = 0; q < 9; ++q) dump_vec(f, m.pml[q]);
  dump_vec(f, m.mloc);
  dump_vec(f, m.m6);
  dump_vec(f, m.mstf);
  dump_vec(f, m.floc);
  dump_vec(f, m.f3);
  dump_vec(f, m.fstf);
  dump_vec(f, m.focloc);
  dump_vec(f, m.focmom);
  dump_vec(f, m.rloc);
  dump_vec(f, m.rpos);
  std::fclose(f);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr,
                 "usage: wavesim_b200 SeisFD3D.conf [--device N] [--steps N] [--out DIR]\n"
                 "                    [--storage f32|f16|bf16] [--dump FILE]\n");
    return 2;
  }
  int device = 0, steps = -1, storage = CGFD_STORE_F32;
  std::string out_dir, dump_path;
  for (int a = 2; a < argc; ++a) {
    const std::string o = argv[a];
    auto next = [&]() -> std::string {
      if (a + 1 >= argc) die("missing value of " + o);
      return argv[++a];
    };
    if (o == "--device") device = std::atoi(next().c_str());
    else if (o == "--steps") steps = std::atoi(next().c_str());
    else if (o == "--out") out_dir = next();
    else if (o == "--dump") dump_path = next();
    else if (o == "--storage") {
      const std::string v = next();
      storage = v == "f16" ? CGFD_STORE_F16 : v == "bf16" ? CGFD_STORE_BF16 : CGFD_STORE_F32;
    } else die("unknown option " + o);
  }
  // SeisFD3D.conf (get_conf in src/simulation.cc:759-790)
  const Par conf(argv[1]);
  const std::string dir = conf.str("seispath");
  if (out_dir.empty()) out_dir = dir;
  Model m;
  m.ni = conf.i("ni");
  m.nj = conf.i("nj");
  m.nk = conf.i("nk");
  m.nt = conf.i("nt");
  m.stept = conf.d("stept");
  m.steph = conf.d("steph");
  if (m.ni < 1 || m.nj < 1 || m.nk < 4 || m.nt < 1 || !(m.stept > 0) || !(m.steph > 0))
    die("bad ni/nj/nk/nt/stept/steph");
  if (m.ni > kMaxCells || m.nj > kMaxCells || m.nk > kMaxCells || m.nt > kMaxSteps)
    die("ni/nj/nk or nt out of range");
  m.N = (size_t)(m.ni + 6) * (m.nj + 6) * (m.nk + 6);
  read_grid(conf, dir, m);
  read_media(conf, dir, m);
  read_absorb(conf, dir, m);
  read_sources(conf, dir, m);
  read_stations(conf, dir, m);
  if (!dump_path.empty()) {
    dump(dump_path, m);
    return 0;
  }
  const int nrun = steps >= 0 ? (steps < m.nt ? steps : m.nt) : m.nt;

  cgfd_desc d;
  std::memset(&d, 0, sizeof(d));
  d.ni = m.ni; d.nj = m.nj; d.nk = m.nk;
  d.steph = m.steph; d.stept = m.stept; d.nt = m.nt;
  d.con_index = m.con; d.hybrid_grid = 1;
  for (int q = 0; q < 6; ++q) d.nabs[q] = m.nabs[q];
  d.storage = storage; d.device = device; d.kernel = CGFD_KERNEL_FUSED;
  cgfd_solver *h = nullptr;
  check(cgfd_create(&d, &h), "cgfd_create");
  check(cgfd_upload_metric(h, m.metric[6].data(), m.metric[7].data(), m.metric[8].data(),
                           m.metric[9].data()), "cgfd_upload_metric", h);
  check(cgfd_upload_media(h, m.alpha.data(), m.beta.data(), m.rho.data()), "cgfd_upload_media", h);
  const double *apd[3] = {m.pml[0].data(), m.pml[1].data(), m.pml[2].data()};
  check(cgfd_upload_pml(h, apd[0], apd[1], apd[2], m.pml[3].data(), m.pml[4].data(),
                        m.pml[5].data(), m.pml[6].data(), m.pml[7].data(), m.pml[8].data()),
        "cgfd_upload_pml", h);
  const int nstf = 2 * (m.nt + 1);
  if (!m.m6.empty())
    check(cgfd_upload_moments(h, (int)m.m6.size() / 6, m.mloc.data(), m.m6.data(), nstf,
                              m.mstf.data()), "cgfd_upload_moments", h);
  if (!m.f3.empty())
    check(cgfd_upload_forces(h, (int)m.f3.size() / 3, m.floc.data(), m.f3.data(), nstf,
                             m.fstf.data()), "cgfd_upload_forces", h);
  if (m.nfoc)
    check(cgfd_upload_focal(h, m.nfoc, m.focloc.data(), m.fnt, m.fdt, m.focmom.data()),
          "cgfd_upload_focal", h);
  if (!m.recv.empty())
    check(cgfd_set_receivers(h, (int)m.recv.size(), m.rloc.data()), "cgfd_set_receivers", h);
  if (m.peakvel) check(cgfd_enable_peak_velocity(h, 1), "cgfd_enable_peak_velocity", h);
  check(cgfd_prepare(h), "cgfd_prepare", h);

  std::vector<SnapWriter> sw;
  for (size_t q = 0; q < m.snaps.size(); ++q) {
    char name[32];
    std::snprintf(name, sizeof(name), "snap_%3.3d.nc", (int)q + 1);
    sw.push_back({join(out_dir, name), &m.snaps[q], {}, 0});
  }
  // step t (0-based) ends with FW at its time; a snapshot with interval tinv
  // is taken after every step t with t % tinv == 0, as SWpick takes FW
  for (int t = 0; t < nrun;) {
    int next = nrun - 1;  // the last step to run in this chunk
    for (const Snap &sn : m.snaps) {
      const int k = ((t + sn.tinv - 1) / sn.tinv) * sn.tinv;  // first multiple >= t
      if (k < next) next = k;
    }
    check(cgfd_step(h, next + 1 - t), "cgfd_step", h);
    t = next + 1;
    for (SnapWriter &w : sw)
      if (next % w.sn->tinv == 0) w.take(h);
  }
  check(cgfd_sync(h, 3600.0), "cgfd_sync", h);
  long long bad = 0;
  cgfd_check_finite(h, &bad);
  if (!m.recv.empty()) {
    std::vector<float> seis((size_t)9 * m.recv.size() * m.nt);
    int done = 0;
    check(cgfd_get_seismograms(h, seis.data(), &done), "cgfd_get_seismograms", h);
    write_seismo(join(out_dir, "seismo.nc"), m, seis, done);
  }
  if (m.peakvel)
    check(cgfd_write_peak_velocity_nc(h, join(out_dir, "peakvel.nc").c_str()),
          "cgfd_write_peak_velocity_nc", h);
  for (const SnapWriter &w : sw) w.write(m.stept);
  std::printf("wavesim_b200: %d x %d x %d cells, %d steps, %zu receivers, %zu snapshots, "
              "%lld non-finite values\n", m.ni, m.nj, m.nk, nrun, m.recv.size(), sw.size(), bad);
  cgfd_destroy(h);
  return bad ? 3 : 0;
}
