/*
 * afid_gpu.h — C ABI of the B200 (sm_100a) implementation of AFiD's RK3 flow + temperature
 * substep.  Plain C types and pointers only; every entry point returns an int status.
 *
 * The reference (chowland/AFiD-MuRPhFi, Fortran 90) runs the path as argument-less
 * subroutines over module state: TimeMarcher (src/flow_solver/TimeMarcher.F90:13) called from
 * the main loop (src/main.F90:306), CalcMaxCFL (src/main.F90:285,350) and CheckDivergence
 * (src/main.F90:249,351).  This ABI replaces those calls: the caller owns the host arrays and
 * builds the metric tables exactly as the reference does (CreateGrid.F90, InitPressureSolver
 * in pressure.F90:61-114); the library owns device buffers and keeps the state resident on
 * the GPU between calls.  The precedent for binding C from the reference is its FFTW
 * interface block (src/flow_solver/param.F90:184-226); a Fortran caller binds these entry
 * points the same way, with an ISO_C_BINDING interface block of bind(C) functions.
 *
 * Array conventions: all 1-D tables are 0-based copies of the reference's 1-based arrays
 * (table[k-1] == fortran(k)).  3-D host arrays are Fortran column-major (x fastest, then y,
 * then z) and are passed as a pointer to element (1,1,1) plus the leading dimensions ld_x
 * (>= nx) and ld_y (>= nym), so arrays with the reference's 2-cell y/z halos
 * (InitVariables.F90:68-73) are passed as &vx(1,1,1) with ld_x = nx, ld_y = nym + 4.
 *
 * Threading: one host thread per context; contexts are independent and may be used from
 * different threads.  No call aborts or throws; errors come back as status codes.
 */
#ifndef AFID_GPU_H
#define AFID_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: the reference's errorcode values where one matches ----------------- */
#define AFID_OK 0
#define AFID_E_ALLOC 8           /* allocation failure (AuxiliaryRoutines.F90:88-91)          */
#define AFID_E_CFL 165           /* CFL*dt > CFLMAX with fixed dt (main.F90:300-302)          */
#define AFID_E_DTMIN 166         /* dt < dtmin with variable dt (main.F90:298)                */
#define AFID_E_DIVERGENCE 169    /* max|div u| > resid (main.F90:357)                         */
#define AFID_E_FFTSIZE 444       /* nym/nzm with a prime factor > 5 (main.F90:272-279)        */
#define AFID_E_SINGULAR 601      /* zero pivot in a Poisson mode (pressure.F90:225-229)       */
#define AFID_E_TIMEOUT 602       /* a bounded device-side wait ran out                        */
#define AFID_E_INVALID 603       /* bad argument / unsupported configuration                  */
#define AFID_E_CUDA 604          /* CUDA runtime error (afid_gpu_cuda_error gives the code)   */
#define AFID_E_CAPACITY 605      /* batch/server slots, HBM budget or a fixed scratch array exhausted */
#define AFID_E_IO 606            /* restart file missing, unreadable or of an unsupported layout */
#define AFID_E_CANCELLED 607     /* a served job cancelled by the caller (afid_serve_cancel)   */

/* precision of the explicit terms and transforms (the implicit solves are always FP64) */
#define AFID_PREC_FP64 0
#define AFID_PREC_MIXED 1        /* FP32 explicit terms, FFTs and pressure transforms        */

typedef struct afid_ctx afid_ctx_t;

/* Grid sizes and metric tables.  Lengths: nx = nxm + 1. */
typedef struct afid_grid {
  int nxm, nym, nzm;             /* cells in x (wall-normal), y, z (periodic)  param.F90:67  */
  double alx3, ylen, zlen;       /* domain size                                 bou.in       */
  const double *xc;              /* [nx]  cell faces       CreateGrid.F90:76, grid.F90:29-53 */
  const double *xm;              /* [nx]  cell centres     CreateGrid.F90:114-117            */
  const double *g3rc;            /* [nx]  face metric      CreateGrid.F90:118-125            */
  const double *udx3c;           /* [nx]  dx/g3rc          CreateGrid.F90:134-138            */
  const double *udx3m;           /* [nxm] dx/d3xc          CreateGrid.F90:134-137            */
  const double *ap3ck, *ac3ck, *am3ck;    /* [nx]  d2/dx2 at faces    CreateGrid.F90:165     */
  const double *ap3sk, *ac3sk, *am3sk;    /* [nxm] d2/dx2, velocity   CreateGrid.F90:171     */
  const double *ap3ssk, *ac3ssk, *am3ssk; /* [nxm] d2/dx2, temperature CreateGrid.F90:177    */
  const double *amphk, *acphk, *apphk;    /* [nxm] Poisson x-coeffs   pressure.F90:103-114   */
  const double *ak1;             /* [nzm] modified wavenumbers in z            pressure.F90:78-86 */
  const double *ak2;             /* [nym] modified wavenumbers in y            pressure.F90:89-97 */
} afid_grid_t;

/* Physics and options (ReadInputFile.F90:109-123, bou.in). */
typedef struct afid_params {
  double ren;                    /* sqrt(|Ra|/Pr)                                             */
  double pect;                   /* ren * Pr                                                  */
  double byct;                   /* buoyancy prefactor (1 unless salinity sets free-fall)     */
  int active_t;                  /* 1 = temperature is buoyant                                */
  int gaxis;                     /* gravity axis 1 (x), 2 (y), 3 (z)                          */
  int inslws, inslwn;            /* no-slip (1) / free-slip (0) lower and upper walls          */
  int tfixs, tfixn;              /* fixed-T (1) / zero-flux (0) lower and upper plates         */
  double xplusu, xminusu;        /* wall velocities (ImplicitAndUpdateVY.F90:54-61)           */
  double dpdy, dpdz;             /* mean pressure gradients; dpdz must be 0 on this path      */
  int nsst;                      /* 3 = RK3 (Rai-Moin), 1 = AB2 (InitTimeMarchScheme.F90)     */
  int precision;                 /* AFID_PREC_FP64 or AFID_PREC_MIXED                         */
  const double *tempbp;          /* [nym*nzm] plate temperature at x = 0 (SetTempBCs.F90), y fastest */
  const double *temptp;          /* [nym*nzm] plate temperature at x = alx3                   */
} afid_params_t;

/* ---- context lifetime ------------------------------------------------------------------ */
/* Replaces InitVariables + InitPressureSolver device-side: allocates the resident state,
 * uploads the tables, plans the FFTs.  State starts at zero. */
int afid_gpu_create(const afid_grid_t *grid, const afid_params_t *params, afid_ctx_t **out);
int afid_gpu_destroy(afid_ctx_t *ctx);
/* Use a caller stream (cudaStream_t passed as void*); NULL restores the context's own. */
int afid_gpu_set_stream(afid_ctx_t *ctx, void *stream);
void *afid_gpu_get_stream(afid_ctx_t *ctx);
int afid_gpu_synchronize(afid_ctx_t *ctx);

/* ---- state transfer -------------------------------------------------------------------- */
/* Copy vx, vy, vz, temp, pr from host (Fortran layout, see top) to the device and zero the
 * RK3 history rux/ruy/ruz/rutemp, as a restart does (ReadFlowInterp.F90:143-171; the
 * history is not saved because rom(1) = 0).  Any pointer may be NULL to leave that field. */
int afid_gpu_upload(afid_ctx_t *ctx, const double *vx, const double *vy, const double *vz,
                    const double *temp, const double *pr, int ld_x, int ld_y);
/* Copy the resident fields back (what WriteFlowField / CalcMeanProfiles need on the host). */
int afid_gpu_download(afid_ctx_t *ctx, double *vx, double *vy, double *vz, double *temp,
                      double *pr, int ld_x, int ld_y);

/* ---- the hot path ---------------------------------------------------------------------- */
/* One full time step: nsst substeps with the reference's gam/rom/alm and beta = dt/ren/2.
 * Replaces `call TimeMarcher` (main.F90:306, TimeMarcher.F90:28-133).  ntime is accepted for
 * call-sequence compatibility (the reference only uses it for the IBM aldto). */
int afid_gpu_timemarcher(afid_ctx_t *ctx, double dt, int ntime);
/* One substep with explicit coefficients (TimeMarcher.F90:38-133 body). */
int afid_gpu_substep(afid_ctx_t *ctx, int ns, double al, double ga, double ro, double dt,
                     double beta);
/* max over cells of |u|/dx summed over directions, at least 1e-8 (CalcMaxCFL.F90:22-46). */
int afid_gpu_cfl(afid_ctx_t *ctx, double *cflm);
/* max over cells of |div u| (CheckDivergence.F90:22-45). */
int afid_gpu_divmax(afid_ctx_t *ctx, double *dmax);
/* Volume Nusselt number, volume-mean kinetic energy and mean temperature, g3rc-weighted as
 * GlobalQuantities.F90:27-80 (nu_vol = 1 + sqrt(Pr|Ra|) <vx T>).  ra_pr = Pr*|Ra|. */
int afid_gpu_globals(afid_ctx_t *ctx, double ra_pr, double *nu_vol, double *ke, double *tmean);

/* ---- diagnostics ------------------------------------------------------------------------ */
const char *afid_gpu_status_string(int status);
int afid_gpu_cuda_error(afid_ctx_t *ctx);   /* last cudaError_t seen by this context */
/* dims = {nxm, nym, nzm, nxmr, nymr, nzmr}; the refined sizes are 0 without salinity. */
int afid_gpu_dims(afid_ctx_t *ctx, int dims[6]);
/* Device pointer and x-stride (elements) of a resident field, for zero-copy interop.
 * which: 0 vx, 1 vy, 2 vz, 3 temp, 4 pr. */
int afid_gpu_field_device_ptr(afid_ctx_t *ctx, int which, void **dptr, int *ldx);
/* Kernels launched by this context since creation (all are this library's own kernels). */
long long afid_gpu_launch_count(afid_ctx_t *ctx);

/* Wall-normal profiles of CalcMeanProfiles.F90 (the means.h5 datasets), computed on the device
 * from the resident state: out[AFID_NUM_PROFILES * nxm], profile q at out + q*nxm, in the order
 * Tbar, vybar, vzbar, vxT, vyT, vzT, Trms, vxrms, vyrms, vzrms, vxvy, vxvz, vyvz, chiT, epsilon. */
#define AFID_NUM_PROFILES 15
int afid_gpu_mean_profiles(afid_ctx_t *ctx, double *out);

/* Spectra of spectra.F90: per (k, ky, kz) the time average of |F|^2, F the y r2c + z c2c
 * Fourier coefficients of vx, vy, vz, temp at k = 1..nxm normalised by 1/(nym nzm).
 * afid_gpu_spectra_update(dt) adds dt*|F|^2 of the resident state (UpdateSpectra, after each
 * TimeMarcher while averaging); afid_gpu_spectra_read(which = 0 vx, 1 vy, 2 vz, 3 temp) gives
 * out[nxm * (nym/2+1) * nzm] (x fastest, then ky, then kz) divided by the accumulated interval
 * (WriteSpectra), *tav = that interval; afid_gpu_spectra_reset starts a new average. */
int afid_gpu_spectra_reset(afid_ctx_t *ctx);
int afid_gpu_spectra_update(afid_ctx_t *ctx, double dt);
int afid_gpu_spectra_read(afid_ctx_t *ctx, int which, double *out, double *tav);
/* One plane of a resident field (which: 0 vx, 1 vy, 2 vz, 3 temp, 4 pr), as the movie cuts
 * write them: axis 0 = x (wall-parallel plane at x index `index`): out[nzm][nym]; axis 1 = y:
 * out[nzm][nx]; axis 2 = z: out[nym][nx]. */
int afid_gpu_slice(afid_ctx_t *ctx, int which, int axis, int index, double *out);
/* Plane mean of a resident field (which: 0 vx, 1 vy, 2 vz, 3 temp) over y (axis 1: out[nzm][nx],
 * ymean of h5tools/means.F90:10-45) or over z (axis 2: out[nym][nx], zmean, means.F90:47-82):
 * the sum over the averaged index in ascending order divided by nym (nzm), on the device. */
int afid_gpu_mean_plane(afid_ctx_t *ctx, int which, int axis, double *out);

/* Autotuner of the fused explicit/implicit kernel: every launch shape available for this
 * wall-normal size (threads per block x rows per thread, register cap, cache policy, columns
 * per block)
 * is timed on a sample of columns, with the RK3 histories redirected to scratch memory so the
 * state is untouched, and the fastest is kept.  It runs by itself before the first step;
 * force = 1 repeats it.  The shape changes the schedule only: results are bitwise the same for
 * every shape. */
#define AFID_TUNE_MAX 8
typedef struct afid_tune_info {
  int ncand;                    /* shapes available (1 = nothing to choose)                  */
  int chosen;                   /* index of the shape in use                                 */
  int sample_columns;           /* x-columns per timed sample launch                         */
  int threads[AFID_TUNE_MAX];   /* threads per column block                                  */
  int rows[AFID_TUNE_MAX];      /* rows per thread                                           */
  int regcap[AFID_TUNE_MAX];    /* registers capped for >= 16 (1) or >= 32 (2) warps per SM  */
  int policy[AFID_TUNE_MAX];    /* bit 0: L1 cache hints (tables kept, streaming data not
                                   allocated); bit 1: two neighbouring columns per block;
                                   bit 2: adjacent rows per thread; bit 3: one persistent block
                                   per SM with the tables in shared memory; bit 4: the first
                                   row's table operands loaded before the staging wait; bit 5:
                                   the CN solves' forward factors loaded before their barrier  */
  double us[AFID_TUNE_MAX];     /* mean time per sample launch in microseconds (-1: not run) */
  int k4_chosen;                /* Poisson tridiagonal: 0 one mode per warp, 1 persistent warps
                                   with the next mode's right-hand side prefetched              */
  double k4_us[2];              /* microseconds per full launch of each form (-1: not run)   */
  int fftz_chosen;              /* z transforms: 0 one tile per block, 1 persistent blocks with
                                   the next tile's copies in flight, 2 the same with the tiles
                                   moved by tensor copies (3-D single domains)                  */
  double fftz_us[3];            /* microseconds per full forward z launch of each form         */
  int ify_chosen;               /* inverse y transform: 0 per-thread copies, 1 tensor copies
                                   (FP64 single domains, nym = 32 x {1,2,3,4,6,8,12})           */
  double ify_us[2];             /* microseconds per full launch of each form (-1: not run)    */
  int div_chosen;               /* divergence + forward y transform: 0 per-thread loads, 1
                                   tensor copies of the velocity rows (FP64 single domains)      */
  double div_us[2];             /* microseconds per full launch of each form (-1: not run)    */
} afid_tune_info_t;
int afid_gpu_autotune(afid_ctx_t *ctx, int force, afid_tune_info_t *info);
/* Use shape `index` (0 .. ncand-1) from now on without timing, e.g. one saved from an earlier
 * afid_gpu_autotune on the same device and sizes.  AFID_E_INVALID for a shape this context
 * cannot run (those the autotuner reports with us = -1 for that reason). */
int afid_gpu_set_k1_shape(afid_ctx_t *ctx, int index);
/* Use Poisson-tridiagonal form `form` (0 or 1 as in afid_tune_info_t.k4_chosen) from now on;
 * both forms give bitwise the same results. */
int afid_gpu_set_k4_form(afid_ctx_t *ctx, int form);
/* Use z-transform form `form` (0, 1 or 2 as in afid_tune_info_t.fftz_chosen); bitwise the same.
 * AFID_E_INVALID for a persistent form whose two tiles of nzm rows do not fit shared memory. */
int afid_gpu_set_fftz_form(afid_ctx_t *ctx, int form);
/* Use inverse-y-transform form `form` (0 or 1 as in afid_tune_info_t.ify_chosen); bitwise the
 * same.  AFID_E_INVALID for form 1 where it does not apply (mixed precision, other nym). */
int afid_gpu_set_ify_form(afid_ctx_t *ctx, int form);
/* Use divergence + forward-y-transform form `form` (0 or 1 as in afid_tune_info_t.div_chosen);
 * bitwise the same.  AFID_E_INVALID for form 1 where it does not apply (mixed precision). */
int afid_gpu_set_div_form(afid_ctx_t *ctx, int form);
/* Test hook of the bounded device waits (no counterpart in the reference).  With polls > 0
 * (at most 2^24), the fused explicit/implicit kernel's staging wait (and those of the
 * tensor-copy transform forms), after its copies have landed, also waits at most `polls` polls for an mbarrier phase that nothing completes: every
 * block gives up, sets the error flag and exits, and the next call that synchronises with the
 * stream (afid_gpu_synchronize, afid_gpu_cfl, afid_gpu_divmax, afid_gpu_globals, ...) returns
 * AFID_E_TIMEOUT.  No fault, no hang; the flag stays set for the life of the context (as the
 * reference stops at its first error code).  polls = 0 restores normal operation. */
int afid_gpu_set_wait_test(afid_ctx_t *ctx, long long polls);
/* Per-kernel device timing with CUDA events recorded on the context stream around every
 * launch (no counterpart in the reference, which times whole steps with MPI_WTIME,
 * main.F90:282,363-371).  Classes: 0 CN factor tables, 1 explicit+implicit, 2 divergence +
 * y FFT, 3 z FFT forward, 4 Poisson tridiagonal, 5 z FFT backward, 6 y FFT backward,
 * 7 projection + pressure update, 8 reductions (CFL, divergence, volume sums), 9 salinity step,
 * 10 salinity interpolation (include/afid_salinity.h). */
#define AFID_PROF_CLASSES 11
int afid_gpu_profile_enable(afid_ctx_t *ctx, int enable);
/* Milliseconds and launch counts per class since the last report; synchronises the stream. */
int afid_gpu_profile_report(afid_ctx_t *ctx, double *ms, long long *count, int n);

/* ---- statistics without allocation -------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library allocate device
 * memory (a host code with its own device pool or a capped allocator, a monitor attached to
 * someone else's run): the same {nu_vol, ke, tmean} as afid_gpu_globals, computed from device
 * fields the caller owns (x-fastest, x-stride ldx >= nxm+1, nym rows per z-plane; g3rc is a
 * device array of nxm values), written to the caller's device array out3[3], stream-ordered on
 * `stream` (cudaStream_t as void*, NULL = legacy default stream).  It calls no allocator: its
 * partial sums live in a static device array of AFID_NOALLOC_SCRATCH_BYTES that every GPU
 * loading this library holds until exit, which limits it to nym*nzm <= 174762 columns
 * (AFID_E_CAPACITY beyond).  The first call on each device looks up that array's address (do
 * it before any stream capture); a device reset or a new context on the device invalidates the
 * address, and the first call after it looks it up again.  Calls share the array and it keeps
 * the last call's contents; calls that overlap on the GPU race.  Each launch's own status is
 * returned (AFID_E_CUDA); errors left by the caller's earlier CUDA calls are not consumed. */
#define AFID_NOALLOC_SCRATCH_BYTES (4u << 20)
int afid_gpu_globals_noalloc(int nxm, int nym, int nzm, int ldx, double alx3, double ra_pr,
                             const double *vx, const double *vy, const double *vz,
                             const double *temp, const double *g3rc, double *out3, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* AFID_GPU_H */
