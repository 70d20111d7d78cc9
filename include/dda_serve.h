/*
 * dda_serve.h -- request loop of the B200 DDA solver (libdda_b200.so).
 *
 * A server owns one device and solves requests (one target, one incidence,
 * one or both polarisations) with continuous batching: requests wait in a
 * queue, are admitted as soon as a worker slot is free and their HBM
 * footprint (dda_footprint) fits the server's budget, and run concurrently,
 * each on its own context and CUDA stream, so the work of requests that
 * arrive while others are on the GPU overlaps on the device.  A request's
 * Krylov state stays on the device from admission to completion.
 *
 * The reference solves one target per process run (ddaMain,
 * DDA/DDAMain.cpp:611-771: geometry, DDAParams, couple constants, incident
 * field, getPolVec, cross sections); one request here is that sequence for
 * one target, without the file output.  The queue, admission and
 * concurrency have no counterpart in the reference.
 *
 * Each request is solved exactly as it would be alone (its own context, the
 * same kernels and reductions), so its result does not depend on what else
 * is in flight.
 */
#ifndef DDA_SERVE_H
#define DDA_SERVE_H

#include <stdint.h>

#include "dda_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dda_server dda_server;

typedef struct dda_serve_request {
  const uint32_t* positions; /* nv*3 grid coordinates, sorted by z (DDA/DDAParams.cpp:441-445) */
  const uint8_t* materials;  /* nv material indices, NULL = all 0 */
  uint32_t nv;
  uint32_t nmat;
  const double* refr;        /* nmat*3 complex refractive indices (x, y, z axis per material) */
  const char* grid_unit;     /* --grid-unit, e.g. "0.1um" (EMSim/Length.cpp syntax) */
  const char* wavelength;    /* --lambda, e.g. "6um" */
  double prop[3];            /* --prop */
  int32_t npol;              /* 1: polarisation 1 only; 2: both */
  int32_t polarizability;    /* DDA_POL_* of dda_frontend.h */
  int32_t solver;            /* DDA_SOLVER_* */
  int32_t precision;         /* DDA_PREC_* */
  double eps;                /* relative residual */
  int64_t max_iter;          /* <= 0: unlimited */
  int32_t keep_pol;          /* 1: keep the polarisations in the result */
  int32_t first_pol;         /* npol == 1: which polarisation (1 or 2; 0 means 1) */
  int32_t grid_policy;       /* DDA_GRID_REFERENCE or DDA_GRID_TUNED (dda_choose_grid) */
  int32_t pad;
  uint64_t tag;              /* caller's label, returned in the result */
} dda_serve_request;

typedef struct dda_serve_result {
  int64_t id;
  uint64_t tag;
  int32_t status;            /* 0 or a DDA_ERR_* code */
  int32_t npol;
  dda_stats stats[2];
  double cext[2], cabs[2];   /* cross sections, m^2 (DDA/Beam.cpp:126-133, DDA/AbsCross.cpp:28-48) */
  double t_submit, t_admit, t_done;  /* seconds on the server clock */
  double t_setup, t_solved;  /* context built (D matrix included); solve finished */
  int64_t footprint;         /* bytes reserved at admission (dda_footprint peak) */
  int64_t device_bytes;      /* bytes the request's context held */
  uint32_t grid[3];
  uint32_t nv;
  int64_t nvs;
  const double* pol;         /* keep_pol: [npol][3][nvs] complex polarisations,
                                valid until dda_serve_release(id) */
  char error[160];
} dda_serve_result;

/* Starts a server on `device` with `max_active` worker slots and an HBM
 * budget in bytes for the admitted requests' contexts (<= 0: 90% of the
 * device memory free at start). */
int dda_serve_create(int device, int64_t hbm_budget, int max_active, dda_server** out);

/* Queues a request (its arrays are copied; the call does not wait for the
 * GPU).  Rejects a request whose footprint exceeds the whole budget. */
int dda_serve_submit(dda_server* s, const dda_serve_request* req, int64_t* id);

/* Moves up to `max` finished results to `out`, waiting up to timeout_ms
 * (< 0: until at least one is ready) for the first; returns how many. */
int dda_serve_poll(dda_server* s, dda_serve_result* out, int max, int timeout_ms);

/* Cancels request `id`.  A queued request leaves the queue at once and its
 * result (status DDA_ERR_CANCELLED) is delivered by dda_serve_poll; a
 * running request's solve stops after its current round of iterations
 * (dda_cancel) and its result reports DDA_ERR_CANCELLED with the iterate
 * reached.  Other requests are not affected.  Returns DDA_ERR_ARG for an id
 * that is neither queued nor running. */
int dda_serve_cancel(dda_server* s, int64_t id);

/* Frees the polarisations kept for result `id`. */
int dda_serve_release(dda_server* s, int64_t id);

/* Requests queued or running. */
int64_t dda_serve_pending(dda_server* s);

/* Seconds since the server started (the clock of the result times). */
double dda_serve_clock(const dda_server* s);

/* Finishes the queued and running requests, then stops the workers. */
int dda_serve_destroy(dda_server* s);

/* Message of the last failed dda_serve_create / dda_serve_submit on this thread. */
const char* dda_serve_error(void);

#ifdef __cplusplus
}
#endif

#endif /* DDA_SERVE_H */
