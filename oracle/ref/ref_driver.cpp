// ref_driver.cpp -- single-process driver for the reference's own device
// runtime (class ChildProcs, src/calculate.cu), used as a parity oracle.
//
// TEST INFRASTRUCTURE ONLY (built by oracle/ref/Makefile into oracle/_ref/).
// It replaces src/simulation.cc for one rank driving one GPU:
//   * builds the cindx exactly as get_conf does (src/simulation.cc:798-835);
//   * writes the par file and device.dat that ChildProcs::GpuAbility reads
//     (src/calculate.cu:2832-2950) into a scratch directory;
//   * fills the public host buffers H_drv, H_mpa, H_apr, H_mnt, H_frc, Hpt,
//     and for the optional outputs and sources HSpt (snapshot points), HFpt
//     and H_Rmnt (focal points and their moment series) (src/typedata.h:
//     148-162), then calls C2DPointPick, C2DSnapPick, C2DFocalPick, ParH2D
//     and VelCoeff in the order of src/simulation.cc:208-228;
//   * runs the time loop of src/simulation.cc:252-700 with the same
//     wavesyn/abssyn/RKite/PWpick/SWpick sequence and direction table.
//     ShareData, IntraBoundGS and BoundGS are not called: with one child rank
//     and one device they only move never-written zeros into the x ghost
//     planes.  With PVflag set, the last stage runs IterationFinalPV and the
//     peak velocities are read from the device buffer Dpv it keeps.
// Input and output are flat binary files (format version 2, see
// oracle/refio.py).  Built with the reference's SrcSmooth option
// (ref_wavesim_smooth) it also reads the sources' smoothing blocks
// (H_mnt.dnorm, H_frc.dnorm) after the input.
#include "typedata.h"

#include <cuda_runtime.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

template <class T>
void rd(FILE *f, T *p, size_t n) {
  if (n && fread(p, sizeof(T), n, f) != n) {
    fprintf(stderr, "ref_driver: short read\n");
    exit(93);
  }
}
template <class T>
void wr(FILE *f, const T *p, size_t n) {
  if (n && fwrite(p, sizeof(T), n, f) != n) {
    fprintf(stderr, "ref_driver: short write\n");
    exit(94);
  }
}

void dl(const Real *dev, std::vector<float> &host, size_t n) {
  host.resize(n);
  if (cudaMemcpy(host.data(), dev, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
    fprintf(stderr, "ref_driver: D2H failed\n");
    exit(95);
  }
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: ref_driver <input.bin> <output.bin> <scratch dir>\n");
    return 2;
  }
  FILE *fi = fopen(argv[1], "rb");
  if (!fi) { perror("input"); return 3; }
  int32_t hdr[28];
  rd(fi, hdr, 28);
  if (hdr[0] != 0x52464743 || hdr[1] != 2) { fprintf(stderr, "bad input header\n"); return 4; }
  const int ni = hdr[2], nj = hdr[3], nk = hdr[4], nt = hdr[5], nsteps = hdr[6];
  const int con = hdr[7];
  int nabs[6];
  for (int q = 0; q < 6; ++q) nabs[q] = hdr[8 + q];
  const int nmnt = hdr[14], nfrc = hdr[15], nstf = hdr[16], nrecv = hdr[17];
  const int has_init = hdr[18], nstages = hdr[19];
  const int write_fields = hdr[20] & 1;
  const int nfoc = hdr[21], fnt = hdr[22], pvflag = hdr[23];
  const int nsnp = hdr[24], snap_tinv = hdr[25] > 0 ? hdr[25] : 1;
  double hd[3];
  rd(fi, hd, 3);
  const Real steph = (Real)hd[0], stept = (Real)hd[1], fdt = (Real)hd[2];

  cindx cdx;
  cdx.ni = ni; cdx.nj = nj; cdx.nk = nk;
  cdx.nx = ni + 2 * LenFD; cdx.ny = nj + 2 * LenFD; cdx.nz = nk + 2 * LenFD;
  cdx.nx1 = 0; cdx.ni1 = LenFD; cdx.ni2 = cdx.ni1 + ni; cdx.nx2 = cdx.ni2 + LenFD;
  cdx.ny1 = 0; cdx.nj1 = LenFD; cdx.nj2 = cdx.nj1 + nj; cdx.ny2 = cdx.nj2 + LenFD;
  cdx.nz1 = 0; cdx.nk1 = LenFD; cdx.nk2 = cdx.nk1 + nk; cdx.nz2 = cdx.nk2 + LenFD;
  const size_t N = (size_t)cdx.nx * cdx.ny * cdx.nz;

  // par file + device file for GpuAbility
  std::string dir = argv[3];
  mkdir(dir.c_str(), 0777);
  char host[256] = {0};
  gethostname(host, 255);
  const std::string conf = dir + "/SeisFD3D.conf";
  {
    FILE *fc = fopen(conf.c_str(), "w");
    fprintf(fc, "BlockPerGrid = 64 32 1\nThreadPerBlock = 256 1 1\n");
    fprintf(fc, "seispath = %s\ndevice_filename = device.dat\n", dir.c_str());
    fclose(fc);
    FILE *fd = fopen((dir + "/device.dat").c_str(), "w");
    fprintf(fd, "used_device_number_%s = 1\ndevice_ydims_%s = 1\nused_device_id_%s = 0\n", host,
            host, host);
    fclose(fd);
  }

  int CSpn[1] = {nsnp};
  ChildProcs cp(conf.c_str(), cdx, steph, stept, nfrc, nmnt, nstf, cdx.nx, ni, 0, con, 1, nabs,
                nrecv, nt, CSpn, nsnp ? 1 : 0, nfoc, nfoc ? fnt : 0, fdt, pvflag, 0, 1, 1);

  rd(fi, cp.H_drv.zetax, N);
  rd(fi, cp.H_drv.zetay, N);
  rd(fi, cp.H_drv.zetaz, N);
  rd(fi, cp.H_drv.jac, N);
  rd(fi, cp.H_mpa.alpha, N);
  rd(fi, cp.H_mpa.beta, N);
  rd(fi, cp.H_mpa.rho, N);
  for (int q = 0; q < 6; ++q) cp.H_apr.nabs[q] = nabs[q];
  rd(fi, cp.H_apr.APDx, cdx.nx); rd(fi, cp.H_apr.APDy, cdx.ny); rd(fi, cp.H_apr.APDz, cdx.nz);
  rd(fi, cp.H_apr.Bx, cdx.nx);   rd(fi, cp.H_apr.By, cdx.ny);   rd(fi, cp.H_apr.Bz, cdx.nz);
  rd(fi, cp.H_apr.DBx, cdx.nx);  rd(fi, cp.H_apr.DBy, cdx.ny);  rd(fi, cp.H_apr.DBz, cdx.nz);
  {
    std::vector<int32_t> loc(3 * nmnt);
    std::vector<float> m6(6 * nmnt);
    rd(fi, loc.data(), loc.size());
    rd(fi, m6.data(), m6.size());
    for (int q = 0; q < nmnt; ++q) {
      cp.H_mnt.locx[q] = loc[3 * q]; cp.H_mnt.locy[q] = loc[3 * q + 1]; cp.H_mnt.locz[q] = loc[3 * q + 2];
      cp.H_mnt.mxx[q] = m6[6 * q]; cp.H_mnt.myy[q] = m6[6 * q + 1]; cp.H_mnt.mzz[q] = m6[6 * q + 2];
      cp.H_mnt.mxy[q] = m6[6 * q + 3]; cp.H_mnt.mxz[q] = m6[6 * q + 4]; cp.H_mnt.myz[q] = m6[6 * q + 5];
    }
    if (nmnt) rd(fi, cp.H_mnt.stf, (size_t)nmnt * nstf);
  }
  {
    std::vector<int32_t> loc(3 * nfrc);
    std::vector<float> f3(3 * nfrc);
    rd(fi, loc.data(), loc.size());
    rd(fi, f3.data(), f3.size());
    for (int q = 0; q < nfrc; ++q) {
      cp.H_frc.locx[q] = loc[3 * q]; cp.H_frc.locy[q] = loc[3 * q + 1]; cp.H_frc.locz[q] = loc[3 * q + 2];
      cp.H_frc.fx[q] = f3[3 * q]; cp.H_frc.fy[q] = f3[3 * q + 1]; cp.H_frc.fz[q] = f3[3 * q + 2];
    }
    if (nfrc) rd(fi, cp.H_frc.stf, (size_t)nfrc * nstf);
  }
  {
    std::vector<int32_t> loc(3 * nrecv);
    rd(fi, loc.data(), loc.size());
    for (int q = 0; q < nrecv; ++q) {
      cp.Hpt.Rsn[q] = q; cp.Hpt.Gsn[q] = q;
      cp.Hpt.locx[q] = loc[3 * q]; cp.Hpt.locy[q] = loc[3 * q + 1]; cp.Hpt.locz[q] = loc[3 * q + 2];
    }
  }
  std::vector<float> init;
  if (has_init) {
    init.resize(9 * N);
    rd(fi, init.data(), init.size());
  }
  {  // focal points: locations, then the moment series [6][nfoc][fnt]
    std::vector<int32_t> loc(3 * nfoc);
    rd(fi, loc.data(), loc.size());
    for (int q = 0; q < nfoc; ++q) {
      cp.HFpt.Rsn[q] = q; cp.HFpt.Gsn[q] = q;
      cp.HFpt.locx[q] = loc[3 * q]; cp.HFpt.locy[q] = loc[3 * q + 1]; cp.HFpt.locz[q] = loc[3 * q + 2];
      cp.H_Rmnt.locx[q] = loc[3 * q]; cp.H_Rmnt.locy[q] = loc[3 * q + 1]; cp.H_Rmnt.locz[q] = loc[3 * q + 2];
    }
    Real *mom[6] = {cp.H_Rmnt.mxx, cp.H_Rmnt.myy, cp.H_Rmnt.mzz,
                    cp.H_Rmnt.mxy, cp.H_Rmnt.mxz, cp.H_Rmnt.myz};
    for (int c = 0; c < 6 && nfoc; ++c) rd(fi, mom[c], (size_t)nfoc * fnt);
  }
  if (nsnp) {  // snapshot points, all nine components every snap_tinv steps
    std::vector<int32_t> loc(3 * nsnp);
    rd(fi, loc.data(), loc.size());
    for (int q = 0; q < nsnp; ++q) {
      cp.HSpt[0].Rsn[q] = q; cp.HSpt[0].Gsn[q] = q;
      cp.HSpt[0].locx[q] = loc[3 * q]; cp.HSpt[0].locy[q] = loc[3 * q + 1];
      cp.HSpt[0].locz[q] = loc[3 * q + 2];
    }
    cp.HSpt[0].tinv = snap_tinv;
    cp.HSpt[0].cmp = 3;
  }
#ifdef SrcSmooth
  // the smoothing blocks of the moments, then of the forces (7^3 each)
  if (nmnt) rd(fi, cp.H_mnt.dnorm, (size_t)nmnt * LenNorm * LenNorm * LenNorm);
  if (nfrc) rd(fi, cp.H_frc.dnorm, (size_t)nfrc * LenNorm * LenNorm * LenNorm);
#endif
  fclose(fi);

  cp.C2DPointPick();
  if (nsnp) cp.C2DSnapPick();
  if (nfoc) cp.C2DFocalPick();
  cp.ParH2D();
  cp.VelCoeff();
  if (has_init) {
    Real *fw[9] = {cp.FW[0].Vx, cp.FW[0].Vy, cp.FW[0].Vz, cp.FW[0].Txx, cp.FW[0].Tyy,
                   cp.FW[0].Tzz, cp.FW[0].Txy, cp.FW[0].Txz, cp.FW[0].Tyz};
    for (int c = 0; c < 9; ++c)
      cudaMemcpy(fw[c], init.data() + (size_t)c * N, N * sizeof(float), cudaMemcpyHostToDevice);
  }

  // direction table of src/simulation.cc:264-641
  static const int dirs[4][4][3] = {
      {{1, 1, 1}, {-1, -1, -1}, {1, 1, 1}, {-1, -1, -1}},
      {{1, 1, -1}, {-1, -1, 1}, {1, 1, -1}, {-1, -1, 1}},
      {{-1, -1, -1}, {1, 1, 1}, {-1, -1, -1}, {1, 1, 1}},
      {{-1, -1, 1}, {1, 1, -1}, {-1, -1, 1}, {1, 1, -1}}};
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<double> step_secs(nsteps, 0.0);
  for (int t = 0; t < nsteps; ++t) {
    const auto ts = std::chrono::steady_clock::now();
    for (int s = 0; s < 4; ++s) {
      if (s == 0) { cp.wavesyn(cp.mW, cp.FW); cp.abssyn(1); }
      else { cp.wavesyn(cp.mW, cp.W); cp.abssyn(2); }
      const int *d = dirs[t % 4][s];
      cp.RKite(s, t, d[0], d[1], d[2]);
    }
    cp.wavesyn(cp.FW, cp.W);
    cp.abssyn(3);
    cp.PWpick(cp.FW, t);
    if (nsnp) cp.SWpick(cp.FW, t);
    cudaDeviceSynchronize();
    step_secs[t] = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
  }
  for (int s = 0; s < nstages; ++s) {  // a partial step after the full ones
    if (s == 0) { cp.wavesyn(cp.mW, cp.FW); cp.abssyn(1); }
    else { cp.wavesyn(cp.mW, cp.W); cp.abssyn(2); }
    const int *d = dirs[nsteps % 4][s];
    cp.RKite(s, nsteps, d[0], d[1], d[2]);
  }
  cudaDeviceSynchronize();
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_driver: CUDA error %s\n", cudaGetErrorString(e));
    return 5;
  }

  FILE *fo = fopen(argv[2], "wb");
  if (!fo) { perror("output"); return 6; }
  int32_t oh[4] = {nrecv, nt, nsteps, nstages};
  wr(fo, oh, 4);
  wr(fo, &secs, 1);
  wr(fo, step_secs.data(), step_secs.size());
  Real *hp[9] = {cp.HPW.Vx, cp.HPW.Vy, cp.HPW.Vz, cp.HPW.Txx, cp.HPW.Tyy,
                 cp.HPW.Tzz, cp.HPW.Txy, cp.HPW.Txz, cp.HPW.Tyz};
  for (int c = 0; c < 9; ++c) wr(fo, hp[c], (size_t)nrecv * nt);
  std::vector<float> buf;
  if (write_fields) {
    wfield sets[2] = {cp.FW[0], cp.W[0]};
    for (auto &w : sets) {
      Real *p[9] = {w.Vx, w.Vy, w.Vz, w.Txx, w.Tyy, w.Tzz, w.Txy, w.Txz, w.Tyz};
      for (int c = 0; c < 9; ++c) {
        dl(p[c], buf, N);
        wr(fo, buf.data(), N);
      }
    }
  }
  if (pvflag) {  // Dpv[0]: [nx][ny], the top valid layer's max |V| per component
    const size_t n2 = (size_t)cdx.nx * cdx.ny;
    Real *pv[3] = {cp.Dpv[0].Vx, cp.Dpv[0].Vy, cp.Dpv[0].Vz};
    for (int c = 0; c < 3; ++c) {
      dl(pv[c], buf, n2);
      wr(fo, buf.data(), n2);
    }
  }
  if (nsnp) {  // HSW[0]: [component][point][time index]
    const size_t ntime = (size_t)((nt + snap_tinv - 1) / snap_tinv);
    wfield &w = cp.HSW[0];
    Real *p[9] = {w.Vx, w.Vy, w.Vz, w.Txx, w.Tyy, w.Tzz, w.Txy, w.Txz, w.Tyz};
    for (int c = 0; c < 9; ++c) wr(fo, p[c], (size_t)nsnp * ntime);
  }
  fclose(fo);
  fflush(stdout);
  _exit(0);  // skip ~ChildProcs: the process ends here
}
