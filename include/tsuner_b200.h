/*
 * tsuner_b200.h -- C ABI of the B200-native TSUNER hot path.
 *
 * Two layers:
 *  1. Drop-in entry points with the reference signatures and return codes:
 *       TSUNER()            replaces TSUNER.h:39 / GPU/main_TSUNER.cu:21
 *       checkCUDAsupport()  replaces TSUNER.h:41 / GPU/CheckCUDASupport.cu:21
 *       initializeGPU()     replaces TSUNER.h:42 / GPU/InitializeGPU.cu:23
 *  2. Fine-grained tsu_* calls (no counterpart in the reference, whose only
 *     interface is the whole-run TSUNER()): create a solver, upload a state,
 *     step it a given number of times, read the state and extrema back.
 *     Tests, bench.py and the ensemble runner use these.
 *
 * All pointers are plain host pointers unless a name says `device`.
 * All calls return an int status (TSU_OK == 0) unless stated otherwise.
 * Nothing here takes or returns framework (torch) types.
 */
#ifndef TSUNER_B200_H
#define TSUNER_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__CUDACC__) || defined(__VECTOR_TYPES_H__)
#include <vector_types.h>
typedef double2 tsu_double2;
#else
/* Same size and alignment as CUDA's double2 (vector_types.h). */
typedef struct tsu_double2 { double x, y; } __attribute__((aligned(16))) tsu_double2;
#endif

#ifndef TSU_NO_SIMPARAMS
/* Layout-identical to `struct SimParams` of TSUNER.h:10-30 (passed by value
 * to TSUNER()).  Units: metres, seconds.  FR is the Chezy coefficient already
 * divided by 8 (Problem_loader.cxx:337-339); Q, Opar, HQB are the derived
 * values of Problem_loader.cxx:340-342. */
typedef struct SimParams {
    double xmin;
    double xmax;
    double ymin;
    double ymax;
    double total_time, save_time;
    int npx, npy, nvol;
    double CFL;
    double Q, R;
    double porosity;
    double DS;
    double FR;
    double Opar;
    double OC;
    double Dsg;
    double HQB;
    double vmax;
    double epsilon_h;
    double dx;
    double dy;
} SimParams;
#endif

/* Status codes.  1 and 2 keep the meaning of the reference TSUNER() return
 * values (GPU/main_TSUNER.cu:20, main_TSUNER.cxx:91-98). */
enum {
    TSU_OK = 0,
    TSU_ERR_GPU_OOM = 1,
    TSU_ERR_HOST_OOM = 2,
    TSU_ERR_INVALID = 3,      /* bad argument / unsupported size or switch */
    TSU_ERR_CUDA = 4,         /* a CUDA runtime call failed */
    TSU_ERR_NO_DEVICE = 5,    /* no usable CUDA device / bad index */
    TSU_ERR_NONFINITE = 6,    /* the device detected a NaN/Inf state */
    TSU_ERR_IO = 7            /* output file could not be written */
};

/* Run-time form of the reference's compile-time switches
 * (Sim_parameters.hxx:45-54).  tsu_switches_default() fills the values the
 * reference ships with. */
typedef struct TsuSwitches {
    int order;        /* 1 | 2                                   (`order`)   */
    int rk;           /* 1 = Runge-Kutta; 0 = MUSCL-Hancock, one stage per
                         step with the half-step predictor of
                         GPU/Reconstructor.cu:280-342 (FP64 form only; the
                         reference marks it "not fully tested")  (`RK`)      */
    int wbc;          /* 0 free | 1 wall | 2 periodic            (`WBC`)     */
    int bedload;      /* 0 | 1                                   (`BEDLOAD`) */
    int suspension;   /* 0 | 1                                   (`SUSPENSION`) */
    int read_files;   /* 1: boundary edges follow the CC series while
                         t < tCC[timeCC-2], then act as walls  (`Read_files`) */
    int bedload_law;  /* 0 = reference Ashida-Michiue law (GPU/SedFlux.cuh:150-168);
                         1 = Grass law q_b = A_g u |u|^2 / (1-p) (no reference
                         counterpart) */
    int precision;    /* 0 = FP64 plain form (bitwise with the reference);
                         1 = FP32 precision form                              */
    double grass_ag;  /* A_g of the Grass law                               */
    double eta0;      /* FP32 form: FP64 still-water level; the free surface is
                         stored as the FP32 deviation eta - eta0 (use the
                         sea level incl. sea-level rise)                      */
    int manning;      /* 1 = the reference's Manning friction branch,
                         GPU/Reconstructor.cu:47-50, as written there: the
                         momentum is MULTIPLIED by c = dt FR^2 |u| / h^(4/3)
                         (the reference marks it "NOT FINISHED, DO NOT USE";
                         a dry cell gives 0/0).  FR is then the data.dat
                         value (no /8, Problem_loader.cxx:337-339).  FP64
                         form only.  0 = Chezy                   (`Manning`) */
    int reserved;     /* 0 */
} TsuSwitches;

/* Per-run constants of the sediment laws, hoisted out of the per-cell code.
 * Each is the exact expression the reference evaluates per cell
 * (GPU/Reconstructor.cu:64-77, GPU/SedFlux.cuh:51-99,150-168), evaluated
 * once on the device so the device pow() is used. */
typedef struct TsuConsts {
    double vs;        /* settling velocity                                  */
    double Rp;        /* particle Reynolds number                           */
    double A_er;      /* alpha1 * pow(Rp, alpha2)                           */
    double sqrt_FR;   /* sqrt(FR)                                           */
    double VP;        /* vs * (1 - porosity)                                */
    double K_dep;     /* 1.64 + 0.4 * pow(DS/Dsg, 1.64)                     */
    double sqrt_OC;   /* sqrt(OC)                                           */
    double DS5;       /* 5 * DS                                             */
} TsuConsts;

typedef struct TsuSolver TsuSolver;

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- drop-in entry points ---------------- */

/* Whole run, as the reference: uploads the state (h, (qx,qy), H; hc = 0),
 * steps while t < params.total_time, writes <input_prefix>.nc with the
 * reference layout (GPU/netcdf.cu:38-435) and the wall time into *tiempo.
 * d, dyrup, time_dyrup, tides_bd, tides_time, tidesNPT are accepted and
 * ignored, as in the reference build (SPL == 0, tides commented out).
 * The switches are the process-wide defaults (tsu_set_default_switches). */
#ifdef __cplusplus
int TSUNER(double *dVh, tsu_double2 *dVhu, double *dVH, int *fixH, SimParams params,
           char *input_prefix, double *d, double *CC, double *tCC, unsigned long timeCC,
           double *dyrup, float *time_dyrup, double &tiempo, int CudaDevice,
           double *tides_bd, float *tides_time, int tidesNPT);
#else
int TSUNER(double *dVh, tsu_double2 *dVhu, double *dVH, int *fixH, SimParams params,
           char *input_prefix, double *d, double *CC, double *tCC, unsigned long timeCC,
           double *dyrup, float *time_dyrup, double *tiempo, int CudaDevice,
           double *tides_bd, float *tides_time, int tidesNPT);
#endif
/* 0 ok, 1 no GPU, 2 no CUDA-capable GPU, 3 bad device index. */
int checkCUDAsupport(int cudaDevice);
/* Creates the CUDA context on the current device (warm-up). */
void initializeGPU(void);

/* ---------------- configuration ---------------- */

int tsu_switches_default(TsuSwitches *sw);
int tsu_set_default_switches(const TsuSwitches *sw);   /* used by TSUNER() */
int tsu_get_default_switches(TsuSwitches *sw);
/* Derived parameters of Problem_loader.cxx:337-342 from the data.dat values
 * (FR given as in data.dat, i.e. before the /8). */
int tsu_derive_params(SimParams *p, double friction_datdat);
/* Parses a reference data.dat (Problem_loader.cxx:264-342 format).  Fills
 * p (xmin..Dsg, derived Q/Opar/HQB, nvol; dx/dy from the box), the output
 * prefix, the three input file names, SLR and the tides file name.  Strings
 * are written NUL-terminated into buffers of `cap` bytes. */
int tsu_parse_data_dat(const char *path, SimParams *p, char *prefix, char *bathy_file,
                       char *ic_file, char *mask_file, double *slr, char *tides_file,
                       size_t cap);

/* ---------------- solver ---------------- */

int tsu_create(TsuSolver **out, const SimParams *p, const TsuSwitches *sw, int device);
int tsu_destroy(TsuSolver *s);
/* Host planes of nvol doubles each, row-major [npy][npx]; hc may be NULL (0). */
int tsu_set_state(TsuSolver *s, const double *h, const double *qx, const double *qy,
                  const double *H, const double *hc);
/* Binary mask (1 = erodible, 0 = fixed), nvol ints, values must be 0 or 1.
 * NULL = all erodible. */
int tsu_set_mask(TsuSolver *s, const int *fixH);
/* Boundary series CC[timeCC][2npx+2npy][4] (eta, u, v, H) and its uniform
 * time axis tCC[timeCC] (interpolations.cxx:368-774 layout). */
int tsu_set_boundary_series(TsuSolver *s, const double *CC, const double *tCC,
                            unsigned long timeCC);
/* Resets t = 0, the running extrema to -1e30 and computes the initial dt
 * (GPU/main_TSUNER.cu:142-149).  Must follow tsu_set_state. */
int tsu_reset(TsuSolver *s);
/* Resume from a checkpoint (no counterpart in the reference, whose NetCDF
 * frames hold derived fields only).  A checkpoint is tsu_get_state,
 * tsu_get_extrema and tsu_get_time of a run; to continue it: tsu_set_state
 * (the saved state), tsu_set_mask, tsu_set_boundary_series, tsu_reset, then
 * tsu_resume with the saved t, step count and extrema (any extrema pointer
 * may be NULL: that field keeps the fresh -1e30).  The next dt is the one
 * tsu_reset computed from the state: the dt the interrupted run would have
 * taken (the same formula on the same state), so an FP64 run continues value
 * for value.  The FP32 form stores surface deviations, which come back
 * through the FP64 state and may then differ in the last float bit;
 * MUSCL-Hancock's working state restarts as the filtered state.
 * TSU_ERR_INVALID before tsu_reset, for a slab, or for t < 0 / steps < 0. */
int tsu_resume(TsuSolver *s, double t, long steps, const double *hmax, const double *bmin_rawH,
               const double *eta_max);
/* Enqueues nsteps time steps on the solver's stream (no host sync). */
int tsu_step(TsuSolver *s, long nsteps);
/* Steps while t < t_end (the reference loop condition), at most max_steps;
 * *steps_done gets the number of steps taken.  Synchronises. */
int tsu_run_until(TsuSolver *s, double t_end, long max_steps, long *steps_done);
/* Waits for the solver's stream, then reports the kernels' status words:
 * TSU_ERR_CUDA when a bounded device wait expired (the step it happened in
 * is unfinished), TSU_ERR_NONFINITE when a cell of the state became NaN or
 * infinite (checked on the last RK stage of every step and by tsu_reset on
 * the uploaded state; the reference has no such check and steps on).  After
 * either, the solver steps again only after tsu_reset (and, for a
 * non-finite state, a new tsu_set_state); until then tsu_step / tsu_run_until
 * return the same code without stepping.  tsu_get_time and tsu_run_until
 * report the same words; TSUNER() returns the code. */
int tsu_sync(TsuSolver *s);
/* 5*nvol doubles SoA (h, qx, qy, H, hc). */
int tsu_get_state(TsuSolver *s, double *V);
int tsu_get_extrema(TsuSolver *s, double *hmax, double *bmin_rawH, double *eta_max);
int tsu_get_time(TsuSolver *s, double *t, double *dt, long *steps);
/* FP32 form only: FP64 sums over the grid after the last step of
 * h (water volume / cell area) and of H + hc (bed + suspended sediment). */
int tsu_get_sums(TsuSolver *s, double *water, double *sediment);
int tsu_get_consts(TsuSolver *s, TsuConsts *k);
/* Device timing of the last tsu_step() call in ms (CUDA events around its
 * kernels; the one-time CUDA-graph build of the first call of 16 or more
 * steps happens before them). */
int tsu_last_step_ms(TsuSolver *s, double *ms);
/* Number of kernel launches the last tsu_step() issued. */
int tsu_last_step_launches(TsuSolver *s, long *launches);
/* Device pointer of the current state (plane-major, row pitch in elements). */
int tsu_state_device(TsuSolver *s, void **ptr, long *pitch_elems, long *plane_elems,
                     int *elem_bytes);
/* ---------------- row slabs of one grid (multi-GPU) ----------------
 * No counterpart in the reference, which runs one grid on one GPU
 * (GPU/main_TSUNER.cu:55).  A grid of p->npy rows is split into row slabs,
 * one per GPU (one process per GPU); a slab owns global rows [j0, j1) and
 * stores two ghost rows on each side that has a neighbour (every side of a
 * periodic grid).  The same fused stage kernels run on the owned rows; the
 * grid's own boundaries (walls, free, the CC series) apply only where a slab
 * has no neighbour, and the series segments and the dt's float rounding use
 * the whole grid.  A step is, per RK stage k: the ghost rows of the buffer
 * the stage reads (k == 0: buffer 0, the state the step starts from;
 * k == 1: buffer 1, the intermediate state) are exchanged with the
 * neighbours (tsu_slab_pack -> transport -> tsu_slab_unpack), then
 * tsu_slab_stage(k); after the last stage the slabs' dt values are reduced
 * to their minimum (tsu_get_dt_device -> MIN all-reduce -> tsu_set_dt_device)
 * -- the grid's dt, since each slab rounds its minimum as the whole grid's.
 * The mask's ghost rows (buffer 2) are exchanged once after tsu_set_mask,
 * and the dt once after tsu_reset.  FP64 plain form, order 2, RK2 only.
 * tsu_set_state / set_mask / get_state / get_extrema take and return the
 * owned rows ([j1 - j0][npx] planes); the boundary series is the whole
 * grid's.  tsu_step / tsu_run_until refuse a slab.  tsuner_b200/slabs.py
 * drives slabs over torch.distributed (NCCL send/recv of the ghost rows into
 * the neighbours' local buffers, no peer loads). */
int tsu_slab_create(TsuSolver **out, const SimParams *p, const TsuSwitches *sw, int j0, int j1, int device);
int tsu_slab_info(TsuSolver *s, int *j0, int *rows, int *ghost_south, int *ghost_north);
/* bytes of one side's message of buffer `which` (0, 1: 5 planes x 2 rows x
 * npx doubles; 2: the mask, 2 rows x npx bytes) */
int tsu_slab_halo_bytes(TsuSolver *s, int which, size_t *bytes);
/* side 0 = south, 1 = north.  pack: the two owned rows next to `side` into
 * the device buffer d_dst ([planes][2][npx], contiguous); unpack: d_src into
 * the two ghost rows beyond `side`.  Both enqueue on the solver's stream. */
int tsu_slab_pack(TsuSolver *s, int which, int side, void *d_dst);
int tsu_slab_unpack(TsuSolver *s, int which, int side, const void *d_src);
/* enqueues RK stage k (0 or 1) of the current step on the owned rows */
int tsu_slab_stage(TsuSolver *s, int k);
/* the next step's dt to / from one device double (stream-ordered copies) */
int tsu_get_dt_device(TsuSolver *s, double *d_dt);
int tsu_set_dt_device(TsuSolver *s, const double *d_dt);
/* issue all further work of the solver on `stream` (a cudaStream_t; NULL is
 * CUDA's legacy default stream), e.g. the stream a communication library
 * uses, so that kernels, copies and messages stay ordered; synchronises the
 * previous stream first */
int tsu_set_stream(TsuSolver *s, void *stream);

/* ---------------- batched ensemble (FP32 form) ----------------
 * No counterpart in the reference (single grid only).  nmembers grids of
 * any sizes (params[i]) with their own switches (sw[i]: precision must be 1
 * and the order the same for all), stepped together: per RK stage one
 * persistent kernel walks the tiles of all members; every member advances
 * with its own dt (segmented min-reduction on the device).  Members are
 * ordinary solvers: fill them through tsu_ens_member() + tsu_set_state /
 * tsu_set_mask / tsu_set_boundary_series, read them back the same way. */
typedef struct TsuEnsemble TsuEnsemble;
int tsu_ens_create(TsuEnsemble **out, int nmembers, const SimParams *params, const TsuSwitches *sw, int device);
int tsu_ens_destroy(TsuEnsemble *e);
int tsu_ens_member(TsuEnsemble *e, int i, TsuSolver **solver);
/* t = 0, extrema and initial dt of every member (after the states are set). */
int tsu_ens_reset(TsuEnsemble *e);
/* Enqueues nsteps steps of every member (no host sync). */
int tsu_ens_step(TsuEnsemble *e, long nsteps);
int tsu_ens_sync(TsuEnsemble *e);
/* Times each tile shape x schedule (static stride / dynamic work counter /
 * one CTA per tile) x resident-CTA count over `steps` steps, keeps the
 * fastest and restores the members' states; optional text report. */
int tsu_ens_autotune(TsuEnsemble *e, int steps, char *report, size_t cap);
int tsu_ens_set_config(TsuEnsemble *e, int variant, int dynamic, int ctas);
int tsu_ens_get_config(TsuEnsemble *e, int *variant, int *tile_x, int *tile_y, int *dynamic, int *ctas,
                       long *ntiles);
int tsu_ens_last_step_ms(TsuEnsemble *e, double *ms);
int tsu_ens_last_step_launches(TsuEnsemble *e, long *launches);
/* Steps every member until its time reaches t_end (members that are done
 * skip their tiles) or max_steps steps were enqueued; *steps_done = steps
 * enqueued.  Members keep their own step counts (tsu_get_time). */
int tsu_ens_run_until(TsuEnsemble *e, double t_end, long max_steps, long *steps_done);

/* ---------------- learned corrector ----------------
 * No counterpart in the reference.  A 6-layer, 32-channel 3x3 convolutional
 * network (BF16 weights and activations, FP32 accumulation on the tensor
 * cores, ReLU between layers) that maps coarse-grid maps (maximum depth,
 * bed change, bathymetry; [3][ny/factor][nx/factor] per sample) plus the
 * fine bathymetry to fine-grid maximum depth and bed change [2][ny][nx]:
 * output = bilinear interpolation of the coarse maps + learned residual.
 * Input channels: the interpolated maps, the fine bathymetry and its
 * sub-grid detail, the coarse wet flag, a constant channel and the cell's
 * column and row, on the fine grid padded by 8 cells of edge values.
 * Trained with Adam on mean-square error against fine solves. */
typedef struct TsuCorrector TsuCorrector;
int tsu_corr_create(TsuCorrector **out, int ny, int nx, int factor, int max_batch, unsigned long long seed,
                    int device);
int tsu_corr_destroy(TsuCorrector *c);
/* fine bathymetry H (depth below datum), [ny][nx] */
int tsu_corr_set_site(TsuCorrector *c, const float *fine_H);
/* appends n samples: coarse [n][3][ny/f][nx/f]; fine [n][2][ny][nx] targets or NULL */
int tsu_corr_add_samples(TsuCorrector *c, int n, const float *coarse, const float *fine);
int tsu_corr_num_samples(TsuCorrector *c, int *n);
/* FP32 master weights [6][32 cout][9 taps][32 cin] and biases [6][32] */
int tsu_corr_get_weights(TsuCorrector *c, float *W, float *B);
int tsu_corr_set_weights(TsuCorrector *c, const float *W, const float *B);
/* iters Adam steps on seeded mini-batches of samples [0, ntrain); loss[iters] (optional) */
int tsu_corr_train(TsuCorrector *c, int ntrain, int iters, int batch, float lr, unsigned long long seed,
                   float *loss);
/* Training and prediction options (defaults 0, 0, 0).  large_residual_weight
 * w (>= 0) weights each pixel's maximum-depth term of the loss by
 * 1 + w * t^2, t = that pixel's normalised target residual, so that the few
 * large residuals at run-up fronts count for more than their share of
 * pixels; clip_depth = 1 clips the corrected maximum depth at 0 (a maximum
 * depth is never negative); envelope k > 0 clamps each predicted residual to
 * k times the largest one that the training pairs of the last
 * tsu_corr_train call needed at that pixel.  TSU_ERR_INVALID for w < 0,
 * clip_depth not 0/1 or k < 0. */
int tsu_corr_set_options(TsuCorrector *c, float large_residual_weight, int clip_depth, float envelope);
/* corrected maps of samples [first, first+n): [n][ny][nx] each; base_* (optional) = interpolation only */
int tsu_corr_predict(TsuCorrector *c, int first, int n, float *out_hmax, float *out_db, float *base_hmax,
                     float *base_db);
/* device time per forward convolution over nimg images and TFLOP/s (the
 * network runs on the fine image padded by 8 cells on each side with its
 * edge values, so that no fine cell sees the convolutions' zero padding;
 * the FLOPs count the padded pixels) */
int tsu_corr_bench_conv(TsuCorrector *c, int nimg, int iters, double *ms_per_conv, double *tflops);
int tsu_corr_last_train_ms(TsuCorrector *c, double *ms, long *convs);
/* Raw kernels on caller-owned device buffers (NHWC BF16, 32 channels):
 * Y = act(conv3x3(X, Wk[cout][tap][cin]) + bias), act = ReLU if relu, then
 * channel n zeroed where gate[p][n] <= 0 (if gate); BF16 (Ybf) or FP32 (Yf)
 * output.  wgrad adds sum_p dZ[p][cout] X[p+off(tap)][cin] to dW[cout][tap][cin]
 * and sum_p dZ[p][cout] to db[cout] (FP32).  stream: cudaStream_t or NULL. */
int tsu_corr_conv3x3(const void *X, int nimg, int H, int W, const void *Wk, const float *bias, int relu,
                     const void *gate, void *Ybf, float *Yf, void *stream);
int tsu_corr_conv3x3_wgrad(const void *X, const void *dZ, int nimg, int H, int W, float *dW, float *db,
                           void *stream);
/* synchronises the device; TSU_ERR_CUDA if a corrector kernel's wait expired */
int tsu_corr_status(void);
const char *tsu_corr_last_error(void);

/* Limit, in nanoseconds, of the kernels' ordinary bounded waits on their own
 * TMA copies and tensor-core MMAs (stage kernels of every form, corrector
 * convolutions) on the CURRENT device; 0 restores the default 0.5 s.  No
 * counterpart in the reference (whose kernels never wait).  It exists so
 * that the error path can be exercised without a GPU fault: with a limit of
 * a few nanoseconds the waits expire while the copies are still in flight,
 * the kernels record the error (tsu_sync / tsu_corr_status report
 * TSU_ERR_CUDA), drain their own copies and MMAs with the full limit, free
 * their tensor memory and return, and the context stays usable.  Call it
 * between steps, with no kernel of the library running. */
int tsu_set_wait_limit_ns(unsigned long long ns);

/* CFL time step of an FP64 state that the caller already holds in device
 * memory, computed without any device allocation by the library.  No
 * counterpart in the reference (its MinReduction works on a buffer that
 * TSUNER() allocates).  It is for callers that cannot let a library call
 * cudaMalloc: a host framework that owns every device byte through its own
 * pool, or a long-running service that forbids allocation after start-up so
 * that its memory use stays fixed.
 * d_h, d_qx, d_qy: device planes of p->npy rows, row pitch `pitch_elems`
 * doubles; d_dt: one device double that receives the step, with the same
 * value tsu_reset() computes (GetDeltaT + MinReduction of the reference,
 * float-rounded above 4096 cells).  `stream` is a cudaStream_t (NULL = the
 * default stream); the call only enqueues work.
 * The per-CTA partial minima live in a fixed file-scope device array of
 * 16384 entries (~128 KiB, held by every GPU that loads the library until
 * exit), so grids above 16384 CTAs of 32 x 8 cells (4,194,304 cells) are
 * rejected with TSU_ERR_INVALID and a message.  The first call on a device
 * looks up the array's device address on that device (make that first call
 * before any stream capture).  The looked-up address is kept for the life of
 * the process, so do not call this entry point again on a device after
 * cudaDeviceReset() there.  Every call shares the array: calls that overlap
 * on the GPU race and must be serialised by the caller.  Failures leave
 * their text in tsu_last_error(). */
int tsu_cfl_dt_noalloc(const double *d_h, const double *d_qx, const double *d_qy, long pitch_elems,
                       const SimParams *p, double *d_dt, void *stream);
/* ---------------- input pipeline (host only) ----------------
 * The arithmetic of the reference's Read_files == 1 loader on grids the
 * caller has already read (the reference reads them from NetCDF4 files,
 * which needs libnetcdf / HDF5): each call restates one reference function,
 * value for value.  Grids are row-major [ny][nx]; geographic coordinates in
 * degrees, NCTR free surface and velocities in centimetres (the reference's
 * UNITS = 0.01).  No device is touched. */
/* interpolate_spherics (interpolations.cxx:779-865): the grid fun
 * [npy_f][npx_f] with first cell centre (xmin_f + dx_f/2, ymin_f + dy_f/2)
 * onto the npx x npy cell centres of [xmin, xmax] x [ymin, ymax] -> sol */
int tsu_nctr_interp_grid(double xmin, double xmax, double ymin, double ymax, double xmin_f, double ymin_f,
                         int npx_f, int npy_f, double dx_f, double dy_f, int npx, int npy, const double *fun,
                         double *sol);
/* fix_eta (interpolations.cxx:867-876), in place */
int tsu_nctr_fix_eta(double *eta, const double *H, int npx, int npy, double slr);
/* interpolate_CC (interpolations.cxx:368-775): boundary series CC
 * [ntime][2npx + 2npy][4] from the NCTR grids ha / ua / va
 * [ntime][nyg][nxg] (grid origin xmin_g, ymin_g, spacing dx_g, dy_g), the
 * simulation box and its bed depth H [npy][npx] */
int tsu_nctr_boundary_series(const double *ha, const double *ua, const double *va, unsigned long ntime, int nxg,
                             int nyg, double xmin_g, double ymin_g, double dx_g, double dy_g, int npx, int npy,
                             double xmin, double xmax, double ymin, double ymax, const double *H, double slr,
                             double *CC);
/* dy_transform + dx_transform (interpolations.cxx:79-94): metres per degree
 * of latitude, per-row east-west spacing dxE[npy], the widest row's width */
int tsu_nctr_sphere_metrics(double ymin, double dy, int npy, double xmax, double xmin, double dx, double *dxE,
                            double *dy_unit, double *dmax);
/* spheric2cartesian (interpolations.cxx:879-968) and spheric2cartesian_CC
 * (:970-1097, in place) */
int tsu_nctr_to_cartesian(double xmin, double xmax, double ymin, double ymax, const double *dxE, double dyE, int npx,
                          int npy, const double *fun, double *sol);
int tsu_nctr_to_cartesian_series(double xmin, double xmax, double ymin, double ymax, const double *dxE, double dyE,
                                 int npx, int npy, unsigned long ntime, double *CC);
/* value assignment (Problem_loader.cxx:576-605): H, h = eta * UNITS + H +
 * slr (clipped at 0), zero discharge, mask = fix >= 0.5 (all 1 without a
 * fix grid) */
int tsu_nctr_assign_state(const double *H_cart, const double *eta_cart, const double *fix_cart, int npx, int npy,
                          double slr, double *h, tsu_double2 *hu, double *H, int *fixH);
/* The whole loader (Problem_loader.cxx:355-625, no sponge layer): bathymetry
 * grid (lon xb[nxb], lat yb[nyb], bathy [nyb][nxb]), optional non-erodible
 * grid (fix NULL: everything erodible), NCTR grids (lon xc, lat yc, times
 * tgrid[ntime], ha / ua / va [ntime][nyc][nxc]) onto an npx x npy grid with
 * sea-level rise slr.  Writes the box and spacing into p (xmin..ymax, dx,
 * dy, npx, npy, nvol), the initial state h, (qx, qy), H, the mask, CC
 * [ntime][2npx+2npy][4] and tCC [ntime]: the inputs of TSUNER(). */
int tsu_nctr_prepare(int nxb, int nyb, const double *xb, const double *yb, const double *bathy, int nxf, int nyf,
                     const double *xf, const double *yf, const double *fix, int nxc, int nyc, const double *xc,
                     const double *yc, unsigned long ntime, const double *tgrid, const double *ha, const double *ua,
                     const double *va, int npx, int npy, double slr, SimParams *p, double *h, tsu_double2 *hu,
                     double *H, int *fixH, double *CC, double *tCC);
/* tides_prep (tides.cxx:170-291): the tide grid [npt][nyt][nxt] (first
 * longitude xp[0]) along the four boundaries -> tides_bd [npt][2npx+2npy];
 * magnitudes above 1e5 become 0.  The reference computes it but its use on
 * the device is commented out (GPU/VolumeSolver.cu:204-214), so TSUNER()
 * accepts and ignores it, as the reference does. */
int tsu_nctr_tides(const double *tides, int nxt, int nyt, unsigned long npt, const double *xp, int npx, int npy,
                   double xmin, double xmax, double ymin, double ymax, double *tides_bd);

/* Bulk host <-> device copies through the library's pinned staging chunks
 * and host worker pool, the path every tsu_set_* / tsu_get_* call of this
 * library uses (the reference copies with plain pageable cudaMemcpy,
 * GPU/main_TSUNER.cu:113-122, :159-162, :199-207).  `nplanes` planes of
 * `rows` rows x `width` bytes; host plane k at host[k] with row pitch
 * `hpitch` bytes, device plane k at dev[k] with row pitch `dpitch` bytes;
 * `device` is the CUDA ordinal that owns the device planes.  Host buffers
 * may be pageable (staged through pinned chunks while host threads fill or
 * drain them) or pinned (copied directly).  Ordered after earlier work on
 * the legacy default stream; synchronous (they return once the bytes have
 * arrived).  TSU_ERR_INVALID for NULL planes or width > pitch. */
int tsu_copy_planes_to_device(int device, int nplanes, void *const *dev, size_t dpitch, const void *const *host,
                              size_t hpitch, size_t width, size_t rows);
int tsu_copy_planes_to_host(int device, int nplanes, void *const *host, size_t hpitch, const void *const *dev,
                            size_t dpitch, size_t width, size_t rows);
int tsu_copy_bytes_to_device(int device, void *dev, const void *host, size_t bytes);
int tsu_copy_bytes_to_host(int device, void *host, const void *dev, size_t bytes);
/* Host worker threads of the copy pool (TSU_HOST_THREADS, default
 * min(cores, 16)); host only, no device use. */
int tsu_host_threads(void);
const char *tsu_strerror(int code);
/* Detail text of the last failing call on this thread ("" if none). */
const char *tsu_last_error(void);
const char *tsu_version(void);
/* sizeof(SimParams), sizeof(TsuSwitches), sizeof(TsuConsts) as compiled
 * into the library, for binding checks (host only, no device use). */
int tsu_struct_sizes(size_t out[3]);

#ifdef __cplusplus
}
#endif
#endif /* TSUNER_B200_H */
