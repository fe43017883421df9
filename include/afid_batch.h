/*
 * afid_batch.h — many independent 2-D convection instances of one size class on one GPU
 * (or one 3-D domain) with the main-loop step control on the device.
 *
 * The reference runs one domain per MPI job (main.F90); there is no batched form in it.  This
 * API advances up to thousands of 2-D Rayleigh-Benard instances together: instances that share
 * nxm, nym and the wall-normal grid (ISTR3, STR3, ALX3; nzm = 1) are stacked in one set of
 * device arrays, every kernel of the substep covers all of them in one launch, and each
 * instance keeps its own Ra, Pr, aspect ratio (YLEN), dt rule (IDTV/DT/CFLMAX/DTMIN/DTMAX of its
 * bou.in), CFL, RK3 history and step counter.  The per-instance step control of main.F90:285-304
 * (CFL -> dt) runs on the device, so a step is a fixed launch sequence captured once in a CUDA
 * graph and replayed.  Instances never exchange data: an instance's result does not depend on
 * which other instances are active in the same batch.
 *
 * A batch created from a bou.in with NZM > 1 holds one 3-D domain (nslots = 1): the same
 * device-side CFL -> dt rule and captured step, so served 3-D jobs run like 2-D slots.
 *
 * Slots: a batch has a fixed number of instance slots; idle slots cost no work.  A slot is
 * (re)configured with afid_batch_configure, loaded with afid_batch_seed or afid_batch_upload,
 * and switched on with afid_batch_set_active.
 */
#ifndef AFID_BATCH_H
#define AFID_BATCH_H

#include <stdint.h>

#include "afid_host.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afid_batch afid_batch_t;

/* Per-instance results of the last completed step. */
typedef struct afid_batch_stat {
  int ntime;        /* steps taken since the slot was loaded */
  int errorcode;    /* 0, 165 (CFL, fixed dt), 166 (dt < dtmin); the instance stops on error */
  double time;      /* simulated time */
  double dt;        /* last dt */
  double cfl;       /* last CFL number (CalcMaxCFL) */
} afid_batch_stat_t;

/* nslots instance slots of the size class of `proto` (nxm, nym, nzm, alx3, istr3, str3); nzm > 1
 * requires nslots = 1.  All slots start configured from `proto`, zero state, inactive, no limit. */
int afid_batch_create(const afid_input_t *proto, int nslots, int precision, afid_batch_t **out);
int afid_batch_destroy(afid_batch_t *b);
int afid_batch_set_stream(afid_batch_t *b, void *stream);
/* Per-slot parameters from a bou.in (Ra, Pr, YLEN, dt rule, walls); the size class must match. */
int afid_batch_configure(afid_batch_t *b, int slot, const afid_input_t *in);
/* Seeded conductive state (afid_initial_temperature) with zero velocity; resets history, time
 * and step counter of the slot. */
int afid_batch_seed(afid_batch_t *b, int slot, uint64_t seed);
/* Host state of one slot in the reference's layout (ld_x >= nx, ld_y >= nym); resets the slot. */
int afid_batch_upload(afid_batch_t *b, int slot, const double *vx, const double *vy, const double *vz,
                      const double *temp, const double *pr, int ld_x, int ld_y);
int afid_batch_download(afid_batch_t *b, int slot, double *vx, double *vy, double *vz, double *temp,
                        double *pr, int ld_x, int ld_y);
/* The slot switches itself off after `nsteps` steps counted from its last load (seed/upload);
 * 0 = no limit.  Lets slots with different step budgets share replayed multi-step chunks. */
int afid_batch_set_limit(afid_batch_t *b, int slot, int nsteps);
/* active[nslots]: nonzero = advance.  Takes effect for the next step. */
int afid_batch_set_active(afid_batch_t *b, const unsigned char *active);
/* nsteps main-loop steps (CFL, dt rule, TimeMarcher) of every active slot; asynchronous on the
 * batch stream (call afid_batch_stats or afid_batch_synchronize to wait). */
int afid_batch_step(afid_batch_t *b, int nsteps);
int afid_batch_synchronize(afid_batch_t *b);
/* stats[nslots] (may be NULL), and per-slot Nu_vol / KE (may be NULL) from GlobalQuantities.F90. */
int afid_batch_stats(afid_batch_t *b, afid_batch_stat_t *stats, double *nu_vol, double *ke);
int afid_batch_num_slots(const afid_batch_t *b);
/* Device bytes the batch holds (for admission control by HBM footprint). */
long long afid_batch_device_bytes(const afid_batch_t *b);
long long afid_batch_launch_count(const afid_batch_t *b);
/* The autotuner of include/afid_gpu.h on this batch's stacked domain (runs by itself before the
 * first captured step). */
int afid_batch_autotune(afid_batch_t *b, int force, afid_tune_info_t *info);
/* Use K1 shape `index` for this batch from now on, as afid_gpu_set_k1_shape (bitwise the same
 * results for every shape). */
int afid_batch_set_k1_shape(afid_batch_t *b, int index);
/* dmax[nslots]: max |div u| of every slot's resident state (CheckDivergence.F90), for the check
 * main.F90:346-358 makes every tout (errorcode 169 above RESID).  The cfl scratch of the step
 * control is reused: not while a step is in flight on the batch stream (it is stream-ordered). */
int afid_batch_divmax(afid_batch_t *b, double *dmax);
/* CalcMeanProfiles.F90 profiles of one slot (layout of afid_gpu_mean_profiles). */
int afid_batch_mean_profiles(afid_batch_t *b, int slot, double *out);

#ifdef __cplusplus
}
#endif
#endif /* AFID_BATCH_H */
