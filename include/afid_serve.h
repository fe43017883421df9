/*
 * afid_serve.h — a request loop for simulation jobs on one GPU (continuous batching).
 *
 * A job is one bou.in (2-D with NZM = 1, or a 3-D domain), a Philox seed for the initial
 * perturbation and a number of main-loop steps.  The server keeps every admitted job's fields
 * resident on the device until it completes.  2-D jobs of one size class share pools (one
 * afid_batch_t per pool, include/afid_batch.h) and 3-D jobs get a pool of their own; a job
 * joins a running pool between chunks, and each slot stops itself on the device after exactly
 * its requested steps (afid_batch_set_limit), so a job's result does not depend on the other
 * jobs in the same launches.
 *
 * Admission is by device-memory footprint: a job is admitted when a free slot of its class
 * exists or a new pool fits in hbm_budget_bytes (idle pools of other classes are released to
 * make room), and, if max_cells_in_flight > 0, when the resident cells of running jobs stay
 * under that cap.  Queue order is FIFO, or shortest job (cells x steps) first.
 *
 * The caller drives the loop: afid_serve_submit as jobs arrive, afid_serve_pump to harvest the
 * pools whose last chunk of chunk_steps has completed, admit queued jobs into pools that are not
 * running, and start the next chunk on every idle pool with jobs (each pool on its own stream;
 * a pump with nothing to do waits for the oldest running chunk), afid_serve_poll for completed
 * results.  One host thread per server; the reference has no served mode (main.F90 runs one job).
 */
#ifndef AFID_SERVE_H
#define AFID_SERVE_H

#include <stdint.h>

#include "afid_host.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afid_server afid_server_t;

enum { AFID_SERVE_FIFO = 0, AFID_SERVE_SHORTEST_FIRST = 1 };

typedef struct afid_serve_config {
  int precision;                  /* AFID_PREC_FP64 or AFID_PREC_MIXED, for every job          */
  long long hbm_budget_bytes;     /* device bytes the server's pools may hold                  */
  int slots_per_pool;             /* 2-D instance slots per pool                               */
  int chunk_steps;                /* steps each pool advances per pump                          */
  long long max_cells_in_flight;  /* cap on cells of running jobs; 0 = device memory only      */
  int policy;                     /* AFID_SERVE_FIFO or AFID_SERVE_SHORTEST_FIRST              */
} afid_serve_config_t;

typedef struct afid_serve_job {
  afid_input_t in;    /* the job's bou.in (dt rule, Ra, Pr, sizes)                              */
  uint64_t seed;      /* Philox seed of the +-1e-3 temperature perturbation (afid_initial_temperature) */
  int nsteps;         /* main-loop steps to run (>= 1)                                          */
  uint64_t tag;       /* caller's id, returned with the result                                  */
  double *temp_out;   /* optional host buffer (nxm+1) x nym x nzm for the final temperature     */
} afid_serve_job_t;

typedef struct afid_serve_result {
  uint64_t tag;
  int errorcode;      /* 0, 165 or 166 (the job stopped at the step that raised it), 607 when
                         cancelled (afid_serve_cancel), or the status that kept it from running
                         (603, 444, or 605 when its pool outgrew the budget after submission) */
  int steps_done;
  double time, dt, cfl, nu_vol, ke;   /* simulated time, last dt and CFL, GlobalQuantities      */
  double t_submit, t_admit, t_done;   /* seconds on the server clock (afid_serve_now)           */
} afid_serve_result_t;

typedef struct afid_serve_status {
  int queued, running, pools;
  long long device_bytes;      /* held by the pools                                            */
  long long cells_in_flight;   /* cells of running jobs                                        */
  long long cell_steps_done;   /* sum over completed jobs of cells x steps                     */
  long long jobs_done;
  int pool_failures;           /* pools taken out after a failed chunk, harvest or launch      */
  int last_cuda_error;         /* cudaError_t behind the last such failure (0: none)           */
} afid_serve_status_t;

int afid_serve_create(const afid_serve_config_t *cfg, afid_server_t **out);
int afid_serve_destroy(afid_server_t *s);
/* Queue a job.  Refused at once, with nothing queued: AFID_E_INVALID if malformed, and
 * AFID_E_CAPACITY if its pool's state arrays alone (the nine FP64 field arrays, the RK3
 * histories, phi and the half spectrum, for 1 slot in 3-D or slots_per_pool slots in 2-D)
 * exceed hbm_budget_bytes.  A queued job that still cannot run comes back as a result with its
 * status in errorcode. */
int afid_serve_submit(afid_server_t *s, const afid_serve_job_t *job);
/* Cancel the job with this tag.  A queued job leaves the queue; a running job stops at the end
 * of its pool's current chunk (its slot is freed; the other jobs of the pool are unaffected).
 * Either way it comes back from afid_serve_poll with errorcode AFID_E_CANCELLED and the steps it
 * ran.  AFID_E_INVALID if no queued or running job has the tag. */
int afid_serve_cancel(afid_server_t *s, uint64_t tag);
/* Harvest completed chunks, admit queued jobs, start the next chunk on idle pools with jobs.
 * A pool whose chunk, harvest or launch fails is taken out on its own: its running jobs come
 * back with the failure's status (AFID_E_CUDA, AFID_E_TIMEOUT, ...) and steps_done 0, the other
 * pools go on, and afid_serve_status counts it (pool_failures, last_cuda_error). */
int afid_serve_pump(afid_server_t *s);
/* Move up to `max` completed results into out[]; *n = how many. */
int afid_serve_poll(afid_server_t *s, afid_serve_result_t *out, int max, int *n);
int afid_serve_status(const afid_server_t *s, afid_serve_status_t *st);
/* Test hook (no counterpart in the reference): the nth next chunk launch of the pump counts as a
 * failed launch (AFID_E_CUDA) without any CUDA call, so that the isolation of a failing pool can
 * be tested without a GPU fault; 0 turns it off. */
int afid_serve_set_fail_test(afid_server_t *s, int nth);
double afid_serve_now(const afid_server_t *s);

#ifdef __cplusplus
}
#endif
#endif /* AFID_SERVE_H */
