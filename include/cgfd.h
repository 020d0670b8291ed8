/*
 * cgfd.h -- C ABI of the B200 (sm_100a) time-stepping solver for the
 * collocated-grid curvilinear finite-difference (CGFD) elastic-wave method.
 *
 * This is the drop-in boundary for the device runtime of CoPara-CGFD3D,
 * i.e. for `class ChildProcs` (src/typedata.h:114-217, implemented in
 * src/calculate.cu).  Every entry point below names the reference interface
 * it replaces.  All functions return an int status (cgfd_status); nothing
 * throws or aborts across this boundary (the reference's CC()/Kcheck() call
 * cudaDeviceReset()+MPI_Abort, src/calculate.cu:17-41).  One solver handle
 * drives one GPU and must be used from one host thread at a time.
 *
 * Index conventions are the reference's (src/simulation.cc:798-835):
 *   full arrays are nx*ny*nz with nx=ni+6, ny=nj+6, nz=nk+6 (LenFD=3 ghost
 *   cells per side), flattened as  g = (i*ny + j)*nz + k  (z fastest);
 *   valid cells have i in [3, ni+3), j in [3, nj+3), k in [3, nk+3);
 *   k grows upwards and k = nk+2 is the free surface.
 * Source and receiver locations are (i,j,k) triples in that index space,
 * exactly like locx/locy/locz of the reference (Cstart = 0, one rank).
 * Field component order is the reference's wfield order
 * (src/typenew.h:265-270): Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz.
 */
#ifndef CGFD_H
#define CGFD_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGFD_ABI_VERSION 1

typedef enum cgfd_status {
    CGFD_OK            = 0,
    CGFD_ERR_ARG       = 1,  /* bad argument, size or index                    */
    CGFD_ERR_CUDA      = 2,  /* CUDA runtime error (text in cgfd_last_error)    */
    CGFD_ERR_STATE     = 3,  /* call out of order (e.g. step before upload)     */
    CGFD_ERR_NOMEM     = 4,  /* device or host allocation failed, or a host     *
                              * thread could not start (a C++ exception inside *
                              * the library, caught at the entry point)        */
    CGFD_ERR_TIMEOUT   = 5,  /* a bounded wait on the device ran out            */
    CGFD_ERR_NONFINITE = 6,  /* NaN or Inf found in the wavefield               */
    CGFD_ERR_NODEVICE  = 7   /* no usable CUDA device                           */
} cgfd_status;

/* Storage type of the 9 wavefields and the RK registers.  Arithmetic is FP32
 * in every case; 16-bit storage keeps one power-of-two scale per field and
 * holds the RK accumulator as its difference from the step state, tW - FW
 * (rounded far more finely than tW itself); cgfd_get_field, cgfd_set_field
 * and cgfd_get_snapshot of CGFD_SET_TW convert, so callers see tW. */
typedef enum cgfd_storage {
    CGFD_STORE_F32  = 0,
    CGFD_STORE_F16  = 1,
    CGFD_STORE_BF16 = 2
} cgfd_storage;

/* Kernel family used for the RK stages. */
typedef enum cgfd_kernel {
    CGFD_KERNEL_FUSED  = 0,  /* z-marching tiled kernel, two x-adjacent cells
                                per thread (default)                       */
    CGFD_KERNEL_SIMPLE = 1,  /* one thread per cell, no tiling (cross-check) */
    CGFD_KERNEL_SCALAR = 2   /* z-marching tiled kernel, one cell per thread
                                (cross-check of the tiled structure)       */
} cgfd_kernel;

/* Field sets that cgfd_get_field / cgfd_set_field address. */
typedef enum cgfd_set {
    CGFD_SET_FW = 0,  /* wavefield at the start of the next step (FW)       */
    CGFD_SET_W  = 1,  /* output of the last RK stage that ran (W)           */
    CGFD_SET_TW = 2   /* RK accumulator (tW)                                */
} cgfd_set;

/* Solver description; fills the role of the ChildProcs constructor arguments
 * (src/calculate.cu:107-111) and of the cindx struct (src/typenew.h:134-141). */
typedef struct cgfd_desc {
    int    ni, nj, nk;   /* valid cells in x, y, z                               */
    double steph;        /* grid spacing h (m); x and y spacing equal h (SimpleCar) */
    double stept;        /* time step (s)                                         */
    int    nt;           /* steps the seismogram buffer holds                     */
    int    con_index;    /* ConIndex: cells with k >= con_index use the full zeta
                            metric, cells below use zeta_z only; 3..nk+2          */
    int    hybrid_grid;  /* HyGrid; must be 1 (default SimpleCar build)           */
    int    nabs[6];      /* CFS-PML widths X1 X2 Y1 Y2 Z1 Z2; Z2 must be 0 (free surface on top) */
    int    storage;      /* cgfd_storage                                          */
    int    device;       /* CUDA device ordinal                                   */
    int    kernel;       /* cgfd_kernel                                           */
} cgfd_desc;

typedef struct cgfd_solver cgfd_solver;

/* Replaces ChildProcs::ChildProcs + device allocation (src/calculate.cu:107-1005).
 * Allocates and zeroes all device state; does not read any file. */
int cgfd_create(const cgfd_desc *desc, cgfd_solver **out);

/* Replaces ChildProcs::~ChildProcs (src/calculate.cu:1007-1334). NULL is a no-op. */
int cgfd_destroy(cgfd_solver *h);

/* Copies the text of the last error of h into buf; with h NULL, the last
 * error of a call without a handle (a failed cgfd_create, the host
 * pre-processing, cgfd_count_nonfinite_noalloc) made by the calling host
 * thread (kept per thread, so concurrent callers do not mix their texts).
 * Replaces the reference's printf diagnostics. */
int cgfd_last_error(const cgfd_solver *h, char *buf, size_t len);

/* Grid metric, FP64, full arrays (nx*ny*nz, reference layout).  Replaces the
 * H_drv buffers + ParH2D (src/typedata.h:148, src/calculate.cu:2050-2115).
 * Under SimpleCar only zeta_{x,y,z} and the Jacobian are used on the device. */
int cgfd_upload_metric(cgfd_solver *h, const double *zeta_x, const double *zeta_y,
                       const double *zeta_z, const double *jac);

/* Media: P velocity (alpha), S velocity (beta), density (rho); full arrays.
 * Replaces H_mpa + ParH2D (src/typedata.h:149, src/calculate.cu:2105-2113).
 * The density of every valid cell must be positive; an upload refused for
 * that (CGFD_ERR_ARG) leaves the solver without media until one succeeds. */
int cgfd_upload_media(cgfd_solver *h, const float *alpha, const float *beta,
                      const float *rho);

/* ADE CFS-PML factors (1-D profiles of length nx, ny, nz): APD = alpha + d/beta,
 * B = beta, DB = d/beta.  Replaces H_apr + ParH2D (src/calculate.cu:2157-2180);
 * the factors come from absorb::CalCFSfactors (src/absorb.cpp:346-805) or from
 * cgfd_cfs_factors below. */
int cgfd_upload_pml(cgfd_solver *h,
                    const double *apd_x, const double *apd_y, const double *apd_z,
                    const double *b_x,   const double *b_y,   const double *b_z,
                    const double *db_x,  const double *db_y,  const double *db_z);

/* Moment-tensor point sources: loc = 3n ints (i,j,k), m6 = 6n floats
 * (mxx myy mzz mxy mxz myz), stf = n*nstf floats sampled every stept/2
 * (nstf >= 2*nt+1).  Replaces H_mnt + ParH2D (src/calculate.cu:2133-2152)
 * and is injected like LoadMoment (src/calculate.cu:6193-6255). */
int cgfd_upload_moments(cgfd_solver *h, int n, const int *loc, const float *m6,
                        int nstf, const float *stf);

/* Single-force point sources: loc = 3n, f3 = 3n (fx fy fz), stf as above.
 * Replaces H_frc + ParH2D and LoadForce (src/calculate.cu:6130-6191). */
int cgfd_upload_forces(cgfd_solver *h, int n, const int *loc, const float *f3,
                       int nstf, const float *stf);

/* Finite-fault (focal) sources: n points at loc (3n ints), each with its own
 * moment time series mom [6][n][fnt] (Mxx, Myy, Mzz, Mxy, Mxz, Myz in N m,
 * the subfault's moment included) sampled every fdt seconds from t = 0.  In
 * every stage each point adds -M(t) / (h^3 J) to the stress RHS at
 * t = (step + tinc/2) * stept, M(t) interpolated linearly between samples
 * and zero outside [0, fdt*(fnt-1)].  Replaces H_Rmnt + InterpFocus /
 * ExtractValue + LoadRmom (src/calculate.cu:2586-2643, 1421-1428,
 * 6257-6319; without the SrcSmooth spreading); the series stay on the
 * device and are interpolated there every stage, where the reference
 * interpolates on the host and copies the values every stage.  n = 0
 * removes them. */
int cgfd_upload_focal(cgfd_solver *h, int n, const int *loc, int fnt, double fdt,
                      const float *mom);

/* Spreads the uploaded sources of one kind (0 moments, 1 forces, 2 focal
 * points) over the 7x7x7 nodes around their nodes, as the reference's
 * SrcSmooth build does in LoadMoment / LoadForce / LoadRmom
 * (src/calculate.cu:6147-6175, 6210-6232, 6275-6296): node (i+a-3, j+b-3,
 * k+c-3) of the source at (i, j, k) takes the fraction weights[q][a][b][c]
 * (n*343 doubles, from cgfd_source_smoothing; the sources' own locations
 * are the block centres), valid nodes only, with that node's J (and rho
 * and the surface factor 2 for forces).  n must equal the uploaded count of
 * that kind; weights = NULL (n = 0) turns the spreading off.  Uploading the
 * sources of the kind again also turns it off. */
int cgfd_set_source_smoothing(cgfd_solver *h, int kind, int n, const double *weights);

/* Receivers (3n ints).  Replaces Hpt + C2DPointPick (src/calculate.cu:2678-2746). */
int cgfd_set_receivers(cgfd_solver *h, int n, const int *loc);

/* Builds the free-surface velocity-gradient matrices in FP64 (the work of
 * VelPDcoeff, src/calculate.cu:3320-3428, called through ChildProcs::VelCoeff,
 * src/calculate.cu:1336-1353) and the per-step CUDA graphs.  Called by
 * cgfd_step on first use; may be called explicitly. */
int cgfd_prepare(cgfd_solver *h);

/* Advances n_steps full RK4 steps with the reference's direction schedule
 * (src/simulation.cc:252-700) and records the receivers after each step
 * (PWpick, src/calculate.cu:2780-2830).  Asynchronous on the solver stream. */
int cgfd_step(cgfd_solver *h, int n_steps);

/* cgfd_step with device timing: *ms receives the CUDA-event time of the
 * n_steps on the solver stream.  When stage_ms is not NULL the steps are
 * issued stage by stage instead of as graphs and *stage_ms receives the mean
 * device time of one RK-stage kernel launch.  No reference counterpart (the
 * reference prints wall-clock progress, src/simulation.cc:710-716). */
int cgfd_step_timed(cgfd_solver *h, int n_steps, float *ms, float *stage_ms);

/* One RK stage exactly as ChildProcs::RKite(RKindex, currT, Xvec, Yvec, Zvec)
 * (src/calculate.cu:1355-1600) followed by the copies the reference's time
 * loop makes around it (wavesyn/abssyn, src/calculate.cu:2956-3119).  After rk_index 3 the
 * step state FW holds the new wavefield.  Receivers are not recorded. */
int cgfd_rk_stage(cgfd_solver *h, int rk_index, int curr_t, int xvec, int yvec,
                  int zvec);

/* Waits (bounded by timeout_s seconds) for all queued work of h. */
int cgfd_sync(cgfd_solver *h, double timeout_s);

/* Number of steps recorded so far. */
int cgfd_steps_done(const cgfd_solver *h, int *n);

/* Seismograms: out = 9 * nrecv * nt floats, laid out like HPW
 * (component-major, then receiver, then time: out[(c*nrecv + r)*nt + t]),
 * recorded from FW after each step.  Replaces PWgather/HPW
 * (src/calculate.cu:2748-2778). */
int cgfd_get_seismograms(cgfd_solver *h, float *out, int *nt_done);

/* Full-array (reference layout) copy of one component of a field set. */
int cgfd_get_field(cgfd_solver *h, int set, int comp, float *out);
int cgfd_set_field(cgfd_solver *h, int set, int comp, const float *in);

/* Counts NaN/Inf values of FW on the device; *n_bad receives the count.
 * Returns CGFD_ERR_NONFINITE when the count is not zero. */
int cgfd_check_finite(cgfd_solver *h, long long *n_bad);

/* Per-component scale exponents of 16-bit storage: a stored value s of
 * component c stands for s * 2^exp2[c] (exact: powers of two).  FP16 storage
 * picks them at cgfd_prepare from the sources and the medium (the estimated
 * peak lands at 2^12 stored units); BF16 keeps them at 0 (its exponent range
 * is FP32's).  Setting them rescales the stored fields so that the values
 * they stand for do not change, and keeps them from then on.  FP32 storage
 * accepts only zeros.  exp2: 9 ints in [-60, 60].
 * No reference counterpart (the reference stores FP32 only). */
int cgfd_set_field_scales(cgfd_solver *h, const int *exp2);
int cgfd_get_field_scales(cgfd_solver *h, int *exp2);

/* NaN/Inf count of any float array on the device (d_values, n values), the
 * same count cgfd_check_finite makes for a solver's wavefield, for callers
 * that cannot call cudaMalloc when they run the check: a host application
 * whose pool owns all device memory, a real-time loop that must not take the
 * allocator's synchronisation, code borrowing another framework's buffers.
 * No reference counterpart (the reference has no NaN/Inf check).
 * It allocates nothing: its scratch is a fixed array in the library's device
 * image, so n is limited to 134,217,728 values per call (larger n returns
 * CGFD_ERR_ARG).  Every call looks up the array's device address (the
 * first call on a device loads the library's device code there, which is
 * set-up work, so it should come before any stream capture).  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * Runs on `stream` (a cudaStream_t, NULL = default stream) and waits for it;
 * returns CGFD_ERR_NONFINITE when *n_bad is not zero. */
int cgfd_count_nonfinite_noalloc(const float *d_values, size_t n, long long *n_bad,
                                 void *stream);
/* The most values cgfd_count_nonfinite_noalloc takes per call (16384 x 8192). */
#define CGFD_NOALLOC_MAX_VALUES 134217728ull

/* -------------------------------- outputs --------------------------------- */

/* Peak ground velocity (the reference's IterationFinalPV / PV_export): when
 * enabled, every step updates max |V| per component at each surface cell
 * (maxima reset to zero on enabling).  out: [3][ni][nj] (valid cells, j
 * fastest). */
int cgfd_enable_peak_velocity(cgfd_solver *h, int on);
int cgfd_get_peak_velocity(cgfd_solver *h, float *out);

/* Sub-volume of a field set (the reference's SWpick/snap_export): reference
 * full-array indices start + n*stride (n < count) per axis; components of
 * comp_mask (bit c = component c) in order; out: [component][i][j][k], k
 * fastest. */
int cgfd_get_snapshot(cgfd_solver *h, int set, const int *start, const int *count,
                      const int *stride, int comp_mask, float *out);

/* The reference's seismo.nc / peakvel.nc variables and dimensions, written
 * as NetCDF classic (64-bit offset) files: seismograms of the steps done
 * (Vx..Tyz [TimeNum][PointNum], currTime, Pnum, Lnum, posx/y/z from pos =
 * 3 floats per receiver or NULL for zeros); peak velocities Vx, Vy, Vz [i][j].
 * The reference writes NetCDF-4 (HDF5); no HDF5 library is used here. */
int cgfd_write_seismograms_nc(cgfd_solver *h, const char *path, const float *pos);
int cgfd_write_peak_velocity_nc(cgfd_solver *h, const char *path);

/* ------------------------ learned absorbing layer ------------------------ */

/* Parameters of the layer's MLP (45 -> 64 -> 64 -> 9, SiLU), FP16, in the
 * order W1 [64][45], b1 [64], W2 [64][64], b2 [64], W3 [9][64], b3 [9]. */
#define CGFD_MLP_PARAMS 7689

/* Enables (weights != NULL) or disables the learned correction of the thin
 * absorbing layer: after every step, each valid cell within `width` cells of
 * an absorbing face (never the free surface) gets a correction of FW from
 * MLP(features), the features being the 9 components at the cell and the
 * next 4 cells along its inward normal, stresses over rho*vp, normalised by
 * their largest magnitude.  The correction of component c at depth d is
 * gains[d][c] * 0.25 * tanh(y_c / 0.25), scaled back the same way and
 * clamped so that it only moves the value toward zero (a learned,
 * state-dependent damping).  Any storage type; members of a batch too.
 * No reference counterpart (the reference has sponge and CFS-PML layers). */
int cgfd_set_boundary_mlp(cgfd_solver *h, int width, const void *weights_fp16);
/* Gains of the correction per depth in the layer (0: the cells next to the
 * domain's edge) and component: gains [width][9], the correction of a cell
 * at depth d, component c is multiplied by gains[d*9+c]; NULL sets all to 1
 * (the default after cgfd_set_boundary_mlp). */
int cgfd_set_boundary_mlp_gains(cgfd_solver *h, const float *gains);
/* The layer's cells (reference indices, 3 ints each), in the order of the
 * features below; *n: capacity in, count out. */
int cgfd_boundary_mlp_cells(cgfd_solver *h, int *ijk, int *n);
/* The current normalised features of the layer's cells (training samples):
 * x [n][45], the per-cell scale and rho*vp. */
int cgfd_boundary_mlp_features(cgfd_solver *h, float *x, float *scale, float *rho_vp);
/* Training: for n samples of features x [n][45] and target outputs t [n][9],
 * the mean over samples of the squared output error and its gradient with
 * respect to the parameters (FP32, CGFD_MLP_PARAMS values), on the current
 * device. */
int cgfd_mlp_gradient(const void *weights_fp16, const float *x, const float *t, int n,
                      float *grad, float *loss);

/* ------------------------------ autotuning ------------------------------- */

/* Tries the work-list shapes of the default kernel family (items per
 * resident CTA 3/6/12/24, shortest z-chunk 12/16/24/32/48 planes, PML cost
 * weight 1/2/3, and the shape in use), times `steps` steps of each (after one
 * warm-up step), keeps the fastest and reports its time per
 * step in *ms_per_step.  The wavefields, auxiliaries, seismograms and step
 * count are saved before and restored after, so the simulation is
 * unchanged; the run needs steps + 1 steps of room in nt and the source time
 * functions, and a second copy of that state in device memory.
 * No reference counterpart (the reference reads BlockPerGrid/ThreadPerBlock
 * from its configuration file). */
int cgfd_autotune(cgfd_solver *h, int steps, float *ms_per_step);
/* The work-list shape in use (after cgfd_prepare, default kernel family):
 * items per resident CTA, shortest z-chunk in planes, PML cost weight of the
 * item order; the autotuner's choice can be read and set on another solver
 * of the same model without tuning again.  No reference counterpart. */
int cgfd_get_work_shape(cgfd_solver *h, int *items_per_cta, int *min_chunk, double *pml_weight);
int cgfd_set_work_shape(cgfd_solver *h, int items_per_cta, int min_chunk, double pml_weight);

/* Test hook of the bounded device waits (no reference counterpart: the
 * reference's waits are cudaDeviceSynchronize calls that abort on error,
 * src/calculate.cu:17-41).  Every mbarrier wait of the default kernel gives
 * up after wait_limit_s (0 < wait_limit_s <= 60) instead of about 2 s, and
 * the velocity part's first CTA does not issue the halo tensor copy of entry
 * `withhold` of its first work item, so its wait for that plane runs out:
 * the CTA records the expiry, drains its own copies (bounded) and returns,
 * and cgfd_sync reports CGFD_ERR_TIMEOUT.  The solver's state is then
 * invalid (destroy it); other solvers are unaffected.  withhold < 0 restores
 * normal operation.  Needs CGFD_KERNEL_FUSED; takes effect from the next
 * step (the step graphs are rebuilt). */
int cgfd_test_withhold_copy(cgfd_solver *h, double wait_limit_s, int withhold);

/* ---------------------- batches of models (one GPU) ----------------------- */

/* A batch steps n independent models (each its own grid, medium, PML,
 * sources, receivers, dt and learned layer; one storage type for all, default
 * kernel family) together.  Launch shape CGFD_BATCH_PERSISTENT (the default):
 * one persistent launch per stage part over every member's work items, so
 * that uneven, small models share the GPU without per-model launch tails.
 * CGFD_BATCH_MEMBERS: every member's own step graphs, each member on its own
 * stream (members that fill the GPU alone run at the single-model kernels'
 * speed).  cgfd_batch_autotune times both shapes (and the work-list shapes of
 * the persistent one) and keeps the fastest.  Each model is a member solver:
 * fill it through the usual upload calls on the handle cgfd_batch_solver
 * returns, read its seismograms and fields there.  All members must be at the
 * same step when the batch steps.
 * No reference counterpart (the reference runs one model per MPI job). */
typedef struct cgfd_batch cgfd_batch;

int cgfd_batch_create(const cgfd_desc *descs, int n, cgfd_batch **out);
int cgfd_batch_solver(cgfd_batch *b, int i, cgfd_solver **h);
int cgfd_batch_prepare(cgfd_batch *b);
int cgfd_batch_step(cgfd_batch *b, int n_steps);
/* n_steps steps timed with CUDA events on the batch's stream (whole batch) */
int cgfd_batch_step_timed(cgfd_batch *b, int n_steps, float *ms);
int cgfd_batch_sync(cgfd_batch *b, double timeout_s);
/* cgfd_autotune for the batch: the shared work list's shapes and the launch
 * shape (for the members shape, every member's own work shape is tuned
 * first); the state and the seismograms are restored afterwards */
int cgfd_batch_autotune(cgfd_batch *b, int steps, float *ms_per_step);
#define CGFD_BATCH_PERSISTENT 0
#define CGFD_BATCH_MEMBERS 1
int cgfd_batch_set_launch(cgfd_batch *b, int shape);
int cgfd_batch_get_launch(cgfd_batch *b, int *shape);
int cgfd_batch_last_error(cgfd_batch *b, char *buf, size_t len);
int cgfd_batch_destroy(cgfd_batch *b);

/* ---------------- host pre-processing helpers (FP64) ---------------------- */

/* Grid node coordinates of the reference's vmap grid type (grid_type =
 * vmap: gridmesh::read_vmapnew, src/gridmesh.cpp:72-533, with smooth_zdepth
 * and set_twoside_space, 1092-1210, and the ghost extension
 * common::interpolated_extend, src/common.cpp:67-130), in FP64.  nsurf
 * interfaces from the top (the surface) down are given per (i, j) column:
 * anchor[((size_t)i*nj + j)*(2 + nsurf) + q] = x, y, z_0 .. z_{nsurf-1}
 * (z decreasing downwards), the content of the reference's <vmap_anchor>
 * block; per layer l = 0..nsurf-2, gridpoints[l] intervals and
 * equalspacing[l] (0: the layer grades its spacing between its
 * neighbours').  hybrid != 0: curvilinear above convers_depth and horizontal
 * planes below, the layers above re-cut in proportion to their thickness as
 * the reference does.  Outputs x, y, z as full arrays (ni+6)(nj+6)(nk+6),
 * z fastest, and *con_index (ConIndex: the first node index of the
 * curvilinear part; 3 when not hybrid).  The reference's input checks apply,
 * and the anchors must be finite (the message is available from
 * cgfd_last_error(NULL, ...)). */
int cgfd_grid_vmap(int ni, int nj, int nk, int nsurf, const int *gridpoints,
                   const int *equalspacing, const double *anchor, int hybrid,
                   double convers_depth, double *x, double *y, double *z, int *con_index);

/* Media of a volume model (the reference's media_type = volume:
 * mediapar::read_volume_new, readdata, volume_discrete, ApplySmooth and
 * MediaStatistics, src/mediaparas.cpp:1273-1424, 2140-2220, 376-440,
 * 1712-1900, and common::equivalence_extend), in FP64: the volume
 * vp / vs / rho [nvx][nvy][nvz] (the model file's Vp, Vs, rho) on increasing
 * axes vx, vy, vz (its x, y and depth variables, compared with the grid's z
 * as they are) is sampled at every grid node (x, y, z: full arrays, as
 * cgfd_grid_vmap makes them) by trilinear interpolation inside the
 * sub-volume that brackets the valid nodes (clamped at its ends); where Vp
 * jumps against a neighbour by >= crit_value or by a fraction >= crit_perc,
 * a valid node takes the average of samp_x * samp_y * samp_z sub-cell
 * samples (density arithmetic, lambda and mu harmonic), when any samp > 1.
 * Outputs alpha (Vp), beta (Vs), rho as full arrays, ghost nodes filled as
 * the reference does, ready for cgfd_upload_media. */
int cgfd_media_volume(int ni, int nj, int nk, const double *x, const double *y, const double *z,
                      int nvx, int nvy, int nvz, const double *vx, const double *vy,
                      const double *vz, const float *vp, const float *vs, const float *rho,
                      double crit_value, double crit_perc, int samp_x, int samp_y, int samp_z,
                      float *alpha, float *beta, float *dens);

/* Volume media model file (the reference's media_filename for media_type
 * = volume, e.g. Vsim_gpu.nc; mediapar::read_volume_new,
 * src/mediaparas.cpp:1273-1425) in NetCDF classic format (CDF-1, -2 or -5;
 * a NetCDF-4 file needs `nccopy -k classic` first): 1-D x, y, depth (or z)
 * axes and Vp, Vs, rho over [x][y][depth], the input of cgfd_media_volume.
 * With vx NULL only *nvx, *nvy, *nvz are set; then vx, vy, vz (n each) and
 * vp, vs, rho (nvx*nvy*nvz each) receive the data. */
int cgfd_read_media_volume_nc(const char *path, int *nvx, int *nvy, int *nvz,
                              double *vx, double *vy, double *vz,
                              float *vp, float *vs, float *rho);

/* Finite-fault series file (the reference's focal_process_NC_file,
 * stf-GPU.nc; source::source / readdata, src/source.cpp:43-56, 796-840) in
 * NetCDF classic format: dimensions NP, NT, global attribute DT (s),
 * Mxx Myy Mzz Mxy Mxz Myz [NP][NT] and posx, posy, posz [NP] (m).  With mom
 * NULL only *np, *nt and *dt are set; then mom receives [6][np][nt] (the
 * layout cgfd_upload_focal takes) and posx/posy/posz the positions.  The
 * reference's simulate_damp factor is not applied. */
int cgfd_read_focal_nc(const char *path, int *np, int *nt, double *dt,
                       double *posx, double *posy, double *posz, float *mom);

/* Grid metric from node coordinates (full arrays, reference layout), by
 * 2-point central differences and cross products, then mirrored into the
 * ghost cells: gridmesh::calmetric (src/gridmesh.cpp:1476-1627).
 * out[0..9] = xi_x xi_y xi_z eta_x eta_y eta_z zeta_x zeta_y zeta_z jac. */
int cgfd_metric_from_coords(int ni, int nj, int nk, double steph,
                            const double *x, const double *y, const double *z,
                            double *const out[10]);

/* ADE CFS-PML profiles: absorb::CalCFSfactors (src/absorb.cpp:346-805).
 * dlx[i] (dly[j], dlz[k]) is steph/|grad xi| at (i, nj1, nk1)
 * (resp. |grad eta| at (ni1, j, nk1), |grad zeta| at (ni1, nj1, k)).
 * Each layer width nabs[f] must lie in [0, n] of its axis (CGFD_ERR_ARG
 * otherwise). */
int cgfd_cfs_factors(int ni, int nj, int nk, const int nabs[6],
                     const double velabs[6], const double bmax[6],
                     const double amax[6], const double *dlx,
                     const double *dly, const double *dlz,
                     double *apd_x, double *apd_y, double *apd_z,
                     double *b_x, double *b_y, double *b_z,
                     double *db_x, double *db_y, double *db_z);

/* Source-time-function types (src/mathfunc.cpp:481-608). */
typedef enum cgfd_stf_type {
    CGFD_STF_GAUSS = 0, CGFD_STF_GAUSS_D = 1, CGFD_STF_RICKER = 2,
    CGFD_STF_RICKER_D = 3, CGFD_STF_BELL = 4, CGFD_STF_BELL_D = 5,
    CGFD_STF_BELL_I = 6, CGFD_STF_STEP = 7
} cgfd_stf_type;

/* Samples an STF n times at spacing dt starting at -start, as
 * source::cal_stf_moment (src/source.cpp:102-131); the reference calls it with
 * dt = stept/2 and n = 2*(nt+1) (src/source.cpp:408,775). */
int cgfd_stf(int type, double start, double t0, double f0, int n, double dt,
             float *out);

/* Nearest valid node of each point (common::reposition,
 * src/common.cpp:225-270, as source::cal_index and seisplot::locpoint use
 * it, src/source.cpp:1040, 1105, 1170, src/seisplot.cpp:412-426): pos = 3n doubles
 * (x, y, z) in the coordinates of x, y, z (full node arrays as for
 * cgfd_metric_from_coords).  A point with z > hyper_height goes to the
 * surface node nearest in x-y and takes that node's z (posz); otherwise the
 * node nearest in 3-D, posz = its own z.  Ties go to the first node in
 * (i, j, k) order.  loc = 3n ints out (full-array indices); posz (n
 * doubles, may be NULL) out. */
int cgfd_locate_points(int ni, int nj, int nk, const double *x, const double *y,
                       const double *z, double hyper_height, int n, const double *pos,
                       int *loc, double *posz);

/* Smoothing weights of the reference's SrcSmooth build (src/source.cpp:
 * 157-378, 1051-1073, 1114-1125, 1203-1214): kind 0 = forces (sub-cell shift
 * from four levels of 3->5 node Lagrange refinement, eighth_locate), kind 1
 * = moment and focal points (shift on a 1/8-index trilinear sub-grid, which
 * also moves loc to the nearest node, MomentShiftPosition).  Then the 7^3
 * Gaussian block (half-width 1.5 nodes) around the shift, normalised to 1,
 * and again over its nodes at or below the surface when it reaches above.
 * pos = 3n (z as cgfd_locate_points returns it), loc = 3n in (from
 * cgfd_locate_points) and out (moved for kind 1), weights = n*343 out,
 * [q][a][b][c] for node (i+a-3, j+b-3, k+c-3). */
int cgfd_source_smoothing(int ni, int nj, int nk, const double *x, const double *y,
                          const double *z, int kind, int n, const double *pos, int *loc,
                          double *weights);

/* Strike/dip/rake (degrees) to a unit moment tensor (mxx myy mzz mxy mxz myz):
 * source::angle2moment (src/source.cpp:134-155). */
int cgfd_angle2moment(double strike, double dip, double rake, double m6[6]);

#ifdef __cplusplus
}
#endif

#endif /* CGFD_H */
