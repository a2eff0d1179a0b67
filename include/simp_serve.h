/* Served request stream over the SIMP hot path on B200 (sm_100a).
 *
 * No reference counterpart: the reference runs one basin per process
 * (simp.f90).  A server keeps the basins of many requests resident in one
 * mixed-precision (or FP64) batch context and advances them together
 * (continuous batching): a request that arrives while others run is admitted
 * as soon as a slot and its share of the device-memory budget are free, and
 * leaves the batch when its step count is reached.  Every spot_every-th
 * request also runs as an FP64 replica in a second batch context, on its own
 * stream, so that the served result can be checked against FP64.
 *
 * Replay model: requests are submitted up front with their arrival times
 * (seconds after the first simp_server_run call); run admits each request
 * no earlier than its arrival, by the wall clock, and returns when every
 * submitted request has completed or failed.
 */
#ifndef SIMP_SERVE_H
#define SIMP_SERVE_H

#include "simp_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct simp_server simp_server;

typedef struct simp_server_config {
    double hbm_budget_bytes;        /* device memory for resident basins        */
    int32_t max_instances;          /* slots of the served batch (<= 1024)       */
    int32_t max_request_particles;  /* largest request accepted                 */
    int32_t quantum_steps;          /* most steps between scheduling decisions  */
    int32_t spot_every;             /* FP64 replica of every k-th request (0: none) */
} simp_server_config;

/* Per-request outcome.  Times are seconds after the start of the run. */
typedef struct simp_request_stats {
    double arrival_s, admitted_s, completed_s;
    int64_t steps;                  /* steps advanced                           */
    int32_t ntotal;
    int32_t status;                 /* SIMP_OK, or the error that retired it    */
    int32_t spot_checked;           /* 1: an FP64 replica ran beside it         */
    int32_t reserved0;
    double err_v, err_h;            /* relative L2 against the FP64 replica     */
} simp_request_stats;

typedef struct simp_server_stats {
    int64_t submitted, completed, failed;
    int64_t cancelled;              /* left by simp_server_cancel               */
    int64_t particle_steps;         /* of completed requests                    */
    int64_t batch_steps;            /* steps of the served batch                */
    int64_t peak_resident_particles;
    int32_t peak_resident_requests;
    int32_t reserved0;
    double makespan_s;              /* run start to the last completion         */
    double capacity_particles;      /* particle capacity the budget gave        */
    double admit_s, step_s, retire_s; /* wall time in admissions, stepping and  */
                                    /* retirements (results out, slots freed)   */
} simp_server_stats;

/* params: the served physics (fixed dt, fixed hsml); its precision is the
 * served form's (SIMP_PREC_MIXED normally).  The budget is split between
 * the served batch and, when spot_every > 0, the FP64 replica batch (room
 * for two of the largest requests). */
SIMP_API int32_t simp_server_create(const simp_params *params, const simp_server_config *cfg,
                                    simp_server **out);
SIMP_API int32_t simp_server_destroy(simp_server *srv);

/* Queues one request (arrays as in simp_gpu_batch_add; they must stay valid
 * until the request completes).  At completion its positions, velocities,
 * thickness and concentration are written to the *_out arrays (2*ntotal,
 * 2*ntotal, ntotal, ntotal; any may be NULL). */
SIMP_API int32_t simp_server_submit(simp_server *srv, const simp_forcing *forcing, int32_t ntotal,
                                    const double *x, const double *vx, const double *mass,
                                    const double *rho, const double *hsml, const double *A,
                                    const double *h, int32_t ntotalb, const double *xb,
                                    const double *massb, int64_t nsteps, double arrival_s,
                                    double *x_out, double *vx_out, double *h_out, double *A_out,
                                    int64_t *request_id);

/* Runs the stream until every submitted request has completed, failed or
 * been cancelled. */
SIMP_API int32_t simp_server_run(simp_server *srv);

/* Cancels a request at the first scheduling decision at or after at_s
 * seconds into the run (at_s < 0: the next decision).  A request still
 * pending is never admitted; a resident one leaves the batch, and its FP64
 * replica, between two steps, with its *_out arrays left untouched; one
 * already completed is not affected.  Its status becomes
 * SIMP_ERR_CANCELLED.  The other requests' results do not change (each is
 * the same as stepped alone).  Safe to call from another thread while
 * simp_server_run runs. */
SIMP_API int32_t simp_server_cancel(simp_server *srv, int64_t request_id, double at_s);

SIMP_API int32_t simp_server_request(const simp_server *srv, int64_t request_id,
                                     simp_request_stats *out);
SIMP_API int32_t simp_server_stats_get(const simp_server *srv, simp_server_stats *out);
SIMP_API const char *simp_server_last_error(const simp_server *srv);

#ifdef __cplusplus
}
#endif

#endif /* SIMP_SERVE_H */
