/*
 * afid_gpu.h -- C-ABI of the B200 implementation of AFiD's RK3 time-step
 * hot path (FP64).
 *
 * The reference (PhysicsofFluids/AFiD, Fortran 90) calls its hot path as
 * argument-less subroutines that share state through the modules `param`,
 * `local_arrays` and `fftw_params` (param.F90:4-177), in the order of
 * TimeMarcher.F90:32-72 and main.F90:167-221.  This library keeps those
 * subroutine boundaries: a *box* holds the state that those modules hold for
 * one simulation (fields, RK history, the shared rhs array's wall row, grid
 * metrics), resident in HBM, and each routine of the reference has an entry
 * point of the same name acting on one box.  Fused entry points advance many
 * boxes at once.
 *
 * Conventions
 *   - Every function returns 0 on success or a negative AFID_E* code; the
 *     text of the last error is returned by afid_last_error().
 *   - Host arrays are FP64 in the reference's Fortran order q(k, j, i), k
 *     (wall-normal x) fastest: nx*nym*nzm values for vx, vy, vz, temp, pr and
 *     the RK history, nxm*nym*nzm for dph.  No halo cells.
 *   - Physics failures do not abort: a box whose step fails carries the
 *     reference's error code in afid_box_scalars.status (165 CFL too large,
 *     166 dt < dtmin, 169 divergence > resid, 266 velocity limit or a
 *     non-finite value; main.F90:184-220) and is skipped by later launches.
 *     Status 1 (AFID_STATUS_HELD) is a box on hold, not a failure.
 *     Status 990 (no counterpart in the reference) marks a box whose
 *     asynchronous tile copy did not complete within the kernel's wait
 *     limit; the kernel stops instead of waiting further.
 *   - One host thread per context; calls on a context are not re-entrant.
 *   - All work is queued on the context's stream; functions that return
 *     host data synchronise that stream.
 */
#ifndef AFID_GPU_H
#define AFID_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AFID_OK 0
#define AFID_EINVAL (-1)    /* bad argument */
#define AFID_ENOMEM (-2)    /* device allocation failed */
#define AFID_ECUDA (-3)     /* CUDA runtime error */
#define AFID_ENOBOX (-4)    /* unknown box id */
#define AFID_EFFT (-5)      /* nym or nzm has a prime factor > 7 (main.F90:156-165, code 444) */
#define AFID_ESIZE (-6)     /* size beyond a fixed limit of the entry point */

/* afid_box_scalars.status of a box on hold (afid_box_set_stop); not an
 * error: afid_box_resume releases it. */
#define AFID_STATUS_HELD 1

/* Largest nym and nzm of a box: one line of either transform, with its
 * twiddles, must fit a block's shared memory. */
#define AFID_MAX_NYZ 3072

typedef struct afid_ctx afid_ctx;

/* Fields a box holds (the arrays of module local_arrays, param.F90:80-87). */
enum afid_field {
  AFID_VX = 0, AFID_VY = 1, AFID_VZ = 2, AFID_TEMP = 3, AFID_PR = 4,
  AFID_RUX = 5, AFID_RUY = 6, AFID_RUZ = 7, AFID_RUTEMP = 8,
  AFID_DPH = 9,            /* nxm rows */
  AFID_QCAP = 10, AFID_DQ = 11, AFID_HRO = 12, AFID_RHS = 13,
  AFID_WALL = 14           /* rhs(1, :, :): nym*nzm values, (j, i) order */
};

/* The bou.in values of one simulation (ReadInputFile.F90:16-56,
 * MANUAL.md).  xc (nx node positions) is passed separately to
 * afid_box_add; afid_make_grid builds it from istr3/str3. */
typedef struct afid_box_params {
  int nxm, nym, nzm;     /* NXM NYM NZM */
  int nsst;              /* 3: RK3, 1: Adams-Bashforth (NSST) */
  double alx3;           /* ALX3D */
  double ylen, zlen;     /* YLEN ZLEN */
  double ray, pra;       /* RA PRA */
  int inslws, inslwn;    /* 1: no-slip, 0: stress-free lower/upper wall */
  double tempbp, temptp; /* plate temperatures (SetTempBCs.F90: 1, 0) */
  double dt;             /* DT: fixed dt, or the first dt when idtv = 1 */
  int idtv;              /* IDTV: 0 fixed dt, 1 CFL-adaptive */
  double cflmax;         /* CFLMAX */
  double dtmin, dtmax;   /* DTMIN DTMAX */
  double vlim;           /* VLIM */
  double resid;          /* RESID (<= 0 disables code 169) */
} afid_box_params;

/* Per-box scalars kept on the device and updated every step. */
typedef struct afid_box_scalars {
  double dt;          /* time step of the last step */
  double time;        /* simulation time */
  double cfl;         /* CalcMaxCFL of the velocity at the start of the last step */
  double cfl_used;    /* cfl*dt (fixed dt) or cfl (variable dt) */
  double divmax;      /* CheckDivergence of the velocity at the start of the last step */
  double vmax[3];     /* max |vz|, |vy|, |vx| (GlobalQuantities.F90:44-46) */
  double nu_bot;      /* CalcPlateNu lower plate, after the last step */
  double nu_top;      /* CalcPlateNu upper plate */
  int ntime;          /* completed steps */
  int status;         /* 0, or the reference error code that stopped this box */
} afid_box_scalars;

/* One per-step record of the device-side history ring (afid_box_history). */
typedef struct afid_step_record {
  double time, dt, cfl_used, divmax, nu_bot, nu_top, vmax_y, vmax_z;
} afid_step_record;

/* ---- library / context ------------------------------------------------ */
int afid_version(void);
const char *afid_last_error(void);
int afid_ctx_create(afid_ctx **ctx, int device);
int afid_ctx_destroy(afid_ctx *ctx);
/* Use an external cudaStream_t (0 reverts to the context's own stream). */
int afid_ctx_set_stream(afid_ctx *ctx, void *stream);
void *afid_ctx_stream(afid_ctx *ctx);
int afid_ctx_synchronize(afid_ctx *ctx);
/* Whether afid_step_graph runs large sets as two halves on two streams of
 * the context (1, the default; AFID_BATCH_STREAMS=1 in the environment makes
 * 0 the default) or whole (0).  A caller that splits its boxes itself, one
 * stream per part, turns it off so that its parts do not share the
 * context's two streams (no counterpart in the reference). */
int afid_ctx_set_split_sets(afid_ctx *ctx, int on);

/* ---- grid and boxes ------------------------------------------------------
 * afid_make_grid: node positions xc(1..nx) of CreateGrid.F90:66-119 for
 * istr3 = 0 (uniform), 4 (tanh), 6 (clipped Chebyshev), plus 7 (pure
 * Chebyshev-Gauss-Lobatto, x_k = alx3 (1 - cos(pi (k-1)/nxm)) / 2). */
int afid_make_grid(int nxm, int istr3, double str3, double alx3, double *xc);
/* Bytes of HBM a box of these parameters holds (for admission control). */
size_t afid_box_device_bytes(const afid_box_params *p);
/* Create a box: allocates its fields (zeroed, as AllocateReal3DArray does,
 * AuxiliaryRoutines.F90:79-97) and computes its metrics (CreateGrid.F90,
 * InitPressureSolver.F90) and time-scheme constants
 * (InitTimeMarchScheme.F90).  nym, nzm <= AFID_MAX_NYZ. */
int afid_box_add(afid_ctx *ctx, const afid_box_params *p, const double *xc, int *box_id);
int afid_box_remove(afid_ctx *ctx, int box_id);
int afid_box_upload(afid_ctx *ctx, int box_id, int field, const double *host);
int afid_box_download(afid_ctx *ctx, int box_id, int field, double *host);
/* The same transfers queued on the context's stream, returning at once (no
 * counterpart in the reference, whose fields live in host memory): the host
 * buffer must stay valid and unchanged (upload) or unread (download) until
 * afid_ctx_synchronize or another call that waits for the stream.  From
 * pinned host memory the copies overlap the caller's other work; transfers of
 * one box are applied in call order. */
int afid_box_upload_async(afid_ctx *ctx, int box_id, int field, const double *host);
int afid_box_download_async(afid_ctx *ctx, int box_id, int field, double *host);
/* Zero the RK history, the carried rhs wall row, time, step count and
 * status; set dt (values <= 0 keep the current dt).  Queued on the
 * context's stream (the host does not wait). */
int afid_box_reset(afid_ctx *ctx, int box_id, double dt);
/* Set the simulation time (the time a restart reads from the continua
 * master record, ReadFlowField.F90:24-40). */
int afid_box_set_time(afid_ctx *ctx, int box_id, double time);
/* Restart onto a new grid (ReadFlowField.F90:63-150 with interp.F90:11-227):
 * ``old`` is one continua dataset (nxo x (nyo-1) x (nzo-1) values in Fortran
 * order, x fastest) of a run with nxo, nyo, nzo points and wall-normal grid
 * istro3/stro3; it is interpolated onto this box's grid (wall-normal grid
 * istr3/str3) and written into ``field`` (AFID_VX, AFID_VY, AFID_VZ or
 * AFID_TEMP) on the device.  As in the reference: at most twice the old
 * points in each direction, istr3 0 or 6 for both grids (the only ones
 * interp.F90's gridnew defines), x grids of extent 1, the field numbering
 * of ReadFlowField (vx regridded on interp's case 1, staggered in z; vz on
 * case 3, staggered in x), faces of the old halo extrapolated linearly,
 * and the stencil of interp.F90:177-191 with three upper-x corners read at
 * the lower x index.  The halo's edges and corners, unset in the
 * reference, are zero.  Allocates a temporary device buffer. */
int afid_box_interp_field(afid_ctx *ctx, int box_id, int field, const double *old, int nxo, int nyo, int nzo,
                          int istro3, double stro3, int istr3, double str3);
int afid_box_get_scalars(afid_ctx *ctx, int box_id, afid_box_scalars *out);
/* afid_box_get_scalars of n boxes with one copy and one wait (no counterpart
 * in the reference): out[q] receives box ids[q]'s record; the set is the
 * same kind of box set afid_step takes. */
int afid_boxes_get_scalars(afid_ctx *ctx, const int *box_ids, int n, afid_box_scalars *out);
/* The same records queued on the context's stream, returning at once (no
 * counterpart in the reference): out[0..n) is filled once the stream gets
 * there (after afid_ctx_synchronize at the latest) and must stay valid
 * until then.  Into pinned host memory the records are written by the
 * device directly (no copy); other memory is filled by a queued copy.
 * Each call's records are those of the boxes at that point of the stream. */
int afid_boxes_get_scalars_async(afid_ctx *ctx, const int *box_ids, int n, afid_box_scalars *out);
/* Hold points of a box (no counterpart in the reference; they move the
 * host's per-step checks of main.F90:207, :256 and :273 onto the device, so
 * that a caller can queue many steps and still stop at the right one).
 * After the step that brings the box's step count to stop_ntime (> 0);
 * with tout > 0, after every step main.F90:207 treats as an output time
 * (the second step, and each step after which mod(time, tout) < dt); and
 * with tmax > 0, after a step that leaves time > tmax: the box is put on
 * hold.  Its status becomes AFID_STATUS_HELD and later launches skip it like
 * a failed box, leaving its fields as that step made them.  Values <= 0
 * disable the respective hold; the setting survives afid_box_reset. */
int afid_box_set_stop(afid_ctx *ctx, int box_id, int stop_ntime, double tout, double tmax);
/* Release a box on hold (status AFID_STATUS_HELD -> 0); a box that is not
 * on hold is left as it is.  Queued on the context's stream. */
int afid_box_resume(afid_ctx *ctx, int box_id);
/* Test switch of the bounded device waits (no counterpart in the
 * reference).  With skip != 0 the z transform of this box arms the
 * mbarrier of each tile slot for the tile's bytes but issues no copy, so
 * its wait runs out: the box gets status 990 and the transform block stops,
 * with no copy in flight; max_polls (> 0) lowers the wait limit of this
 * box's tiles (0: the built-in limit).  skip = 0, max_polls = 0 restore
 * normal operation. */
int afid_box_test_skip_z_copies(afid_ctx *ctx, int box_id, int skip, unsigned max_polls);
/* Launch-shape tuning of one box (no counterpart in the reference):
 * row pairs per y-FFT block and ky columns per z-FFT block (powers of two;
 * 0 = built-in choice) and the variant of the explicit/forward kernel:
 * 2 = 32x8-column tiles, two resident blocks per SM; 3 = 32x8, three
 * resident blocks; 4 = 32x8, two planes per barrier; 5, 7, 8 = 32x4 tiles,
 * four, five or six blocks; 6 = 32x2 tiles, eight blocks (0 = 4).  Results
 * do not depend on these values. */
int afid_box_set_tuning(afid_ctx *ctx, int box_id, int fft_y_lines, int fft_z_lines, int k1_minb);
/* Copies up to max_records of the most recent per-step records, oldest
 * first; returns the number copied (>= 0) or an error code. */
int afid_box_history(afid_ctx *ctx, int box_id, afid_step_record *out, int max_records);

/* ---- routine-level entry points (one box) --------------------------------
 * Each replaces the reference subroutine of the same name.  The substep
 * coefficients al, ga, ro, beta (TimeMarcher.F90:22-30) are set by
 * afid_time_marcher_begin_substep from the box's dt. */
int afid_time_marcher_begin_substep(afid_ctx *ctx, int box_id, int ns);  /* TimeMarcher.F90:22-30 */
int afid_explicit_terms_vx(afid_ctx *ctx, int box_id);       /* ExplicitTermsVX.F90:11 */
int afid_explicit_terms_vy(afid_ctx *ctx, int box_id);       /* ExplicitTermsVY.F90:11 */
int afid_explicit_terms_vz(afid_ctx *ctx, int box_id);       /* ExplicitTermsVZ.F90:11 */
int afid_explicit_terms_temp(afid_ctx *ctx, int box_id);     /* ExplicitTermsTemp.F90:11 */
int afid_implicit_and_update_vx(afid_ctx *ctx, int box_id);  /* ImplicitAndUpdateVX.F90:14 + SolveImpEqnUpdate_X.F90:12 */
int afid_implicit_and_update_vy(afid_ctx *ctx, int box_id);  /* ImplicitAndUpdateVY.F90:14 + SolveImpEqnUpdate_YZ.F90:12 */
int afid_implicit_and_update_vz(afid_ctx *ctx, int box_id);  /* ImplicitAndUpdateVZ.F90:14 + SolveImpEqnUpdate_YZ.F90:12 */
int afid_implicit_and_update_temp(afid_ctx *ctx, int box_id);/* ImplicitAndUpdateTemp.F90:13 + SolveImpEqnUpdate_Temp.F90:11 */
int afid_calc_local_divergence(afid_ctx *ctx, int box_id);   /* CalcLocalDivergence.F90:12 */
int afid_solve_pressure_correction(afid_ctx *ctx, int box_id); /* SolvePressureCorrection.F90:12 */
int afid_correct_velocity(afid_ctx *ctx, int box_id);        /* CorrectVelocity.F90:11 */
int afid_correct_pressure(afid_ctx *ctx, int box_id);        /* CorrectPressure.F90:11 */
int afid_calc_max_cfl(afid_ctx *ctx, int box_id, double *cflm);      /* CalcMaxCFL.F90:11 */
int afid_check_divergence(afid_ctx *ctx, int box_id, double *qmax);  /* CheckDivergence.F90:11 */
int afid_calc_plate_nu(afid_ctx *ctx, int box_id, double *nuslow, double *nusupp); /* CalcPlateNu.F90:11 */

/* ---- fused fast path over a set of boxes ---------------------------------
 * afid_step: nsteps passes of main.F90:171-200 (CalcMaxCFL, dt rule,
 * TimeMarcher, time += dt, CalcPlateNu) for every listed box, each kernel
 * launched once for all boxes.  afid_step_graph does the same through a
 * CUDA graph of one step, captured on first use per box set.  A set of at
 * least 8 boxes and 4 Mi cells runs there as two halves of about equal
 * cells, each with its own graph on a stream of the context, forked from
 * and joined back to the context's stream (afid_ctx_set_split_sets); the
 * results are the same either way. */
int afid_step(afid_ctx *ctx, const int *box_ids, int nbox, int nsteps);
int afid_step_graph(afid_ctx *ctx, const int *box_ids, int nbox, int nsteps);
/* Kernels one afid_step_graph step of this set launches (both halves of a
 * split set); captures the graphs if needed (no counterpart in the
 * reference). */
int afid_step_graph_kernels(afid_ctx *ctx, const int *box_ids, int nbox, int *kernels);
/* One substep ns of TimeMarcher.F90:28-72 with the current dt (no CFL). */
int afid_substep(afid_ctx *ctx, const int *box_ids, int nbox, int ns);

/* Kernel slots of afid_step_profiled. */
enum afid_kernel {
  AFID_K_DIAG = 0,          /* CalcMaxCFL + CheckDivergence + vmax reduction */
  AFID_K_FINALIZE = 1,      /* dt rule / step bookkeeping */
  AFID_K_PREP = 2,          /* substep coefficients and x-tridiagonal LU */
  AFID_K_EXPLICIT_FWD = 3,  /* ExplicitTerms* + ImplicitAndUpdate* rhs + forward sweeps */
  AFID_K_IMPLICIT_BWD = 4,  /* back substitution + update of vx, vy, vz, temp */
  AFID_K_FFT_Y_FWD = 5,     /* r2c along y */
  AFID_K_FFT_Z_FWD = 6,     /* c2c along z, forward */
  AFID_K_POISSON_X = 7,     /* complex tridiagonal per (ky, kz) */
  AFID_K_FFT_Z_INV = 8,     /* c2c along z, backward */
  AFID_K_FFT_Y_INV = 9,     /* c2r along y into dph */
  AFID_K_CORRECT = 10,      /* CorrectVelocity + CorrectPressure */
  AFID_K_PLATE_NU = 11,     /* CalcPlateNu partial sums */
  AFID_K_DIVERGENCE = 12,   /* CalcLocalDivergence */
  AFID_K_COUNT = 13
};
/* afid_step with a CUDA event after every launch: adds each kernel's
 * device time (ms) into kernel_ms[slot] and its launch count into
 * kernel_launches[slot] (may be NULL); nkernel >= AFID_K_COUNT. */
int afid_step_profiled(afid_ctx *ctx, const int *box_ids, int nbox, int nsteps,
                       double *kernel_ms, int *kernel_launches, int nkernel);

/* ---- output-time diagnostics (main.F90:202-216) ---------------------------
 * Called between steps at output times, as main.F90 does.  Each call reads
 * the box's current vx, vy, vz and temp once on the device; sums run in a
 * fixed order (results do not depend on scheduling). */
typedef struct afid_global_q {
  double nu_vol;          /* 1 + sqrt(Pr Ra) <T vx> (nu_vol.out) */
  double vmax[3];         /* max |vz|, |vy|, |vx| */
  double tempm, tempmax, tempmin;
  double vz_rms, vy_rms, vx_rms, vel_rms;   /* rms_vel.out, times sqrt(Ra/Pr) */
} afid_global_q;
int afid_global_quantities(afid_ctx *ctx, int box_id, afid_global_q *out);  /* GlobalQuantities.F90:11 */
/* Profiles accumulated per box (module stat_arrays), AFID_NSTAT x nxm values,
 * profile by profile: CalcStats adds the first nine and increments the
 * sample count; CalcDissipationNu adds disste and dissth. */
enum afid_stat {
  AFID_STAT_VX_ME = 0, AFID_STAT_VY_ME, AFID_STAT_VZ_ME, AFID_STAT_TEMP_ME,
  AFID_STAT_VX_RMS, AFID_STAT_VY_RMS, AFID_STAT_VZ_RMS, AFID_STAT_TEMP_RMS,
  AFID_STAT_TEMPVX_ME, AFID_STAT_DISSTE, AFID_STAT_DISSTH, AFID_NSTAT
};
int afid_calc_stats(afid_ctx *ctx, int box_id);                               /* StatRoutines.F90:12 */
int afid_calc_dissipation_nu(afid_ctx *ctx, int box_id, double *nu_mu, double *nu_th); /* CalcDissipationNu.F90:11 */
int afid_box_get_stats(afid_ctx *ctx, int box_id, double *out, int *nstatsamples);
int afid_box_reset_stats(afid_ctx *ctx, int box_id);
/* kslab(1..9) of InitializeSlabDump (SlabDumpRoutines.F90:42-67) from the
 * eight x positions of stst3.in (host only, 1-based k). */
int afid_slab_locations(int nxm, const double *xc, const double *xslab, int *kslab);
/* SlabDumper (SlabDumpRoutines.F90:11-35): for each of nslab (<= 16) 1-based
 * planes, (vx(k)+vx(k+1))/2, vy(k), vz(k), temp(k) as nym x nzm arrays in
 * (j, i) order: out holds nslab*4*nym*nzm doubles. */
int afid_slab_dump(afid_ctx *ctx, int box_id, const int *kslab, int nslab, double *out);

/* ---- pressure solve without allocation ------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they run (memory handed to their own pool, code paths where
 * cudaMalloc is not allowed, a fixed device footprint): the pressure solve of
 * afid_solve_pressure_correction on a dph array the caller owns, with all
 * scratch in one fixed device array inside the library (about 48.5 MiB, held
 * on every GPU that loads the library until exit).  No cudaMalloc, cudaFree or
 * other allocating call is made.
 *   dph    device pointer, in/out: nxm*nym*nzm doubles in the library's
 *          device layout dph[k][i][j] (y fastest, then z, then x), 16-byte
 *          aligned (as every cudaMalloc result is)
 *   xc     host pointer: the nx = nxm+1 node positions
 *   stream cudaStream_t to queue the work on (0: the default stream)
 *   status NULL, or a host int: the call then waits for its work and stores
 *          the status word, 0 or 990 when a transform's tile copy did not
 *          complete within the kernel's wait limit (dph is then not to be
 *          trusted); without it the call returns after queueing the work
 * Limits: nxm <= 1024, nym and nzm <= 3072 (nym even, prime factors <= 7),
 * nxm*nzm*(nym/2+1) <= 2^21; larger boxes return AFID_ESIZE.
 * The first call on a device looks up the array's device address.  Each
 * call stages its small per-call data through host memory that the next
 * call reuses, so a call on a stream that is being captured into a CUDA
 * graph is refused (AFID_EINVAL).  All calls share the array and find the
 * previous call's contents in it; calls that overlap on the GPU race, so the
 * caller must not run two at once. */
int afid_solve_pressure_correction_noalloc(double *dph, int nxm, int nym, int nzm,
                                           const double *xc, double alx3, double ylen,
                                           double zlen, void *stream, int *status);

#ifdef __cplusplus
}
#endif
#endif /* AFID_GPU_H */
