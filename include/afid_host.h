/*
 * afid_host.h — host-side drop-in pieces around the GPU substep (C ABI, plain C types).
 *
 * These replace the reference's set-up and step control that surround TimeMarcher:
 *   afid_parse_bou_in / afid_read_bou_in  ReadInputFile.F90:20-123 (same fixed bou.in layout)
 *   afid_tables_create                    CreateGrid.F90:11-179 + grid.F90 + InitPressureSolver
 *                                         (pressure.F90:61-114) + SetTempBCs.F90:18-41, producing
 *                                         the afid_grid_t / afid_params_t that afid_gpu_create takes
 *   afid_initial_temperature              seeded conductive profile + perturbation
 *                                         (CreateInitialConditions.F90:178-201, RNG replaced)
 *   afid_next_dt                          dt rule and CFL checks of main.F90:285-304
 *   afid_run                              the main loop main.F90:281-422 (CFL, dt, TimeMarcher,
 *                                         divergence check, exit codes) on the GPU
 */
#ifndef AFID_HOST_H
#define AFID_HOST_H

#include <stdint.h>

#include "afid_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afid_input {
  int nxm, nym, nzm, nsst;
  int multires, nxmr, nymr, nzmr;
  int flagsal, flagpf;
  int nread, ireset;
  int ntst;
  double walltimemax, tmax;
  double tout, tframe, save_3d;
  double alx3, ylen, zlen;
  int istr3;
  double str3;
  int istr3r;
  double rayt, prat, rays, pras;
  int ffscales;
  int idtv;
  double dt, resid, limit_cfl, dtmin, dtmax;
  int inslws, inslwn, tfixs, tfixn, sfixs, sfixn;
  int active_t, active_s, gaxis;
  double xplusu, xminusu, dpdy, dpdz;
  int melt;
} afid_input_t;

typedef struct afid_tables afid_tables_t;

int afid_parse_bou_in(const char *text, afid_input_t *out);
int afid_read_bou_in(const char *path, afid_input_t *out);
/* precision: AFID_PREC_FP64 / AFID_PREC_MIXED, copied into the params view */
int afid_tables_create(const afid_input_t *in, int precision, afid_tables_t **out);
void afid_tables_destroy(afid_tables_t *t);
const afid_grid_t *afid_tables_grid(const afid_tables_t *t);
const afid_params_t *afid_tables_params(const afid_tables_t *t);
/* named 1-D table (e.g. "xm", "udx3c", "ap3sk", "ak2"); NULL if unknown; *len set */
const double *afid_tables_array(const afid_tables_t *t, const char *name, int *len);

/* Philox4x32-10 uniform in [0,1) for counter n and key seed (53-bit mantissa) */
double afid_philox_uniform(uint64_t seed, uint64_t n);
/* temp(k,j,i) = T_b + (T_t - T_b) xm_k / alx3 + amp_k (2U - 1), amp_k = eps clamped at the walls,
 * U keyed by n = k + nx*(j + nym*i) (0-based); Fortran layout with leading dims ld_x, ld_y. */
int afid_initial_temperature(const afid_tables_t *t, uint64_t seed, double eps, double *temp,
                             int ld_x, int ld_y);
/* main.F90:287-304: updates *dt, returns 0 / 165 / 166 */
int afid_next_dt(const afid_input_t *in, int ntime, double *dt, double cflm, double *cfl_report);

typedef struct afid_run_stats {
  int steps_done;
  int errorcode;          /* 0, 165, 166, 169, 333 (tmax), 555 (ntst reached) */
  double time, dt, cfl, divmax;
  double nu_vol, ke;      /* at the end of the run */
  double seconds;         /* wall time of the step loop */
} afid_run_stats_t;

/* Run nsteps steps (or ntst+1 if nsteps < 0) of the main loop from the seeded initial
 * condition.  Optional per-step callback gets (step, time, dt, nu_vol, ke) every
 * stats_every steps (0 = never). */
typedef void (*afid_step_cb)(int ntime, double time, double dt, double nu_vol, double ke, void *user);
int afid_run(const afid_input_t *in, int precision, uint64_t seed, int nsteps, int stats_every,
             afid_step_cb cb, void *user, afid_run_stats_t *stats);

#ifdef __cplusplus
}
#endif
#endif /* AFID_HOST_H */
