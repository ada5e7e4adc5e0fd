/*
 * le2d.h -- extensions of the le2d task API (B200 implementation).
 *
 * Everything here is new surface: the reference (le2d `simple/le_core.h`) has no
 * device, so it has no explicit host/device sync, no error query and no batched
 * or served solves.  All functions return an LE2D_* status (0 = ok) unless stated.
 */
#ifndef LE2D_H
#define LE2D_H

#include <stddef.h>
#include "le_core.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define LE2D_OK 0
#define LE2D_EINVAL 1     /* bad argument (sizes < 3, steps < 0, CFL > 1, NULL, ...) */
#define LE2D_ENOTASK 2    /* task->grid was not made by le_init_task of this library */
#define LE2D_ESTYPE 3     /* le_step on an ST_SOA task or le_step_soa on an ST_AOS task */
#define LE2D_ECUDA 4      /* a CUDA call failed (message on stderr) */
#define LE2D_ENOMEM 5     /* device or host allocation failed */
#define LE2D_ENODEV 6     /* no CUDA device */
#define LE2D_EBUDGET 7    /* request does not fit the HBM budget */
#define LE2D_ETIMEOUT 8   /* a bounded wait on the device gave up */
#define LE2D_ESTATE 9     /* call not allowed in the current state */

const char *le2d_strerror(int code);

/* Select the CUDA device used by later calls from this thread (default: device 0).
 * Tasks stay on the device that was current when le_init_task made them. */
int le2d_set_device(int device);

/* Sticky per-task status: the first error since le_init_task / le2d_clear_error. */
int le2d_last_error(const le_task *task);
int le2d_clear_error(le_task *task);

/* Copy the device state to task->grid and wait (the reference grid is then current). */
int le2d_sync_host(le_task *task);
/* The caller wrote task->grid directly: upload it before the next step. */
int le2d_sync_device(le_task *task);
/* Wait for every queued step of the task. */
int le2d_wait(le_task *task);

/* Replace the device state with `src` (5*n.x*n.y reals in the task's layout, any host
 * memory; page-locked memory copies fastest).  task->grid is left untouched. */
int le2d_upload(le_task *task, const real *src);
/* Copy the current state into `dst` (task layout) and wait; task->grid is left untouched. */
int le2d_download(le_task *task, real *dst);

/* Page-locked host memory for le2d_upload / le2d_download buffers (NULL on failure). */
void *le2d_host_alloc(size_t bytes);
void le2d_host_free(void *p);

/* nsteps time steps in one call (le_step semantics for ST_AOS, le_step_soa for ST_SOA);
 * long runs are replayed from a captured CUDA graph. */
int le2d_step_n(le_task *task, int nsteps);
/* As le2d_step_n, and reports the device time of the steps (CUDA events on the task's
 * stream, synchronised), in milliseconds. */
int le2d_step_n_timed(le_task *task, int nsteps, float *ms);

/* Step kernels: FUSED = x- and y-sweep fused per strip, one or two steps per launch;
 * SPLIT = the plain scheme, one kernel per sweep. */
#define LE2D_METHOD_FUSED 0
#define LE2D_METHOD_SPLIT 1
int le2d_set_method(le_task *task, int method);

/* Fused-kernel variant (columns per lane / register bound / input-ring depth / temporal-block
 * depth / warp pair; -1 = default) and row segment length (0 = the planner's) for this
 * task's grid.  A variant of temporal-block depth 2 advances two steps per launch; odd step
 * counts and le_step_soa then take single steps.  On a warp-pair variant a wait between the
 * two warps of a tile that runs out (a fault, not a slow partner) is reported as
 * LE2D_ETIMEOUT at the next synchronisation (le2d_wait, le2d_download, le2d_sync_host). */
int le2d_set_variant(le_task *task, int variant, int seg_len);
/* out[8] = {variant, columns per lane, segment rows, strips, tiles, blocks,
 * temporal-block depth, warps per tile (2: producer / consumer warp pair)}. */
int le2d_get_plan(const le_task *task, int *out);
/* *parts = kernel launches per fused launch of the grid: 1, or 3 when the task's launches go
 * in halves (the band of rows around the middle row on a high-priority stream and the rows
 * above and below it on two more streams, waiting for each other only where their stencils
 * meet -- chosen per grid and plan where it measured faster; LE2D_HALVES=1 / 0 forces it on
 * / off for tasks created afterwards). */
int le2d_launch_parts(const le_task *task, int *parts);

/* Autotuner: times every compiled fused-kernel variant (columns per lane, register bound,
 * input-ring depth, temporal-block depth, warp pair) and row-segment length on a scratch
 * state of nx x ny nodes, and keeps
 * the fastest for the size class (nx, ny rounded up to powers of two).  Tasks created
 * afterwards in that class use it; with LE2D_AUTOTUNE=1 le_init_task tunes a class on its
 * first task.  out_plan (may be NULL) as le2d_get_plan; *nu_per_s (may be NULL) = the
 * measured node-updates/s of the chosen plan. */
int le2d_autotune(int nx, int ny, int *out_plan, double *nu_per_s);
/* Forgets every tuned size class. */
int le2d_autotune_reset(void);

/* Simulated time and step count since le_init_task (FP64 accumulator). */
int le2d_sim_time(const le_task *task, double *t, long long *steps);

/* FP64 diagnostics of the current state: elastic energy (h.x*h.y * sum of
 * rho/2|v|^2 + strain energy), per-field sum of squares and max |value|. */
typedef struct {
	double energy;
	double sumsq[5];
	double maxabs[5];
} le2d_diag_t;
int le2d_diagnostics(le_task *task, le2d_diag_t *out);

/* The same diagnostics for callers that cannot allocate device memory -- hosts that
 * budget every byte of device memory up front (a fixed serving arena), or time loops
 * where a cudaMalloc/cudaFree would synchronise the device.  No counterpart in the
 * reference (which has no device and no diagnostics).  Needs no task and allocates
 * nothing: d_state is the caller's SoA state on the current device (field k, row j,
 * column i at d_state[k*plane + j*pitch + i]; pitch >= nx, plane >= pitch*ny), `stream`
 * a cudaStream_t (NULL = legacy default stream), result in *out.  Its scratch is a
 * library-static device array of per-row partial sums (reduced in a fixed order, so
 * repeated calls give identical results) for at most LE2D_DIAG_NOALLOC_MAX_ROWS rows
 * (larger grids: LE2D_EINVAL); every GPU that loads the library holds it (~1.4 MB)
 * until exit.  All calls share it: calls whose kernels overlap on the GPU race.  The
 * first call on a device (and the first after a reset of that device) looks up the
 * array's device address; make that first call before any stream capture.  Each call
 * synchronises `stream` before it returns (it reads the result back to *out). */
#define LE2D_DIAG_NOALLOC_MAX_ROWS 16384
int le2d_diagnostics_noalloc(const real *d_state, int nx, int ny, long long pitch,
			     long long plane, real hx, real hy, real c1, real c2, real rho,
			     void *stream, le2d_diag_t *out);

/* ---- Batched solves ------------------------------------------------------------------
 * Many independent solves of different sizes, materials, initial conditions and step
 * counts, advanced together by one persistent kernel over a tile work list (each tile
 * carries its instance's material, h and dt).  The step loop runs in windows of
 * `window_steps` steps captured in a CUDA graph. */
typedef struct {
	int nx, ny;            /* grid size, >= 3 each */
	real hx, hy;           /* spacing */
	real dt;               /* time step */
	real c1, c2, rho;      /* material (le_init_material) */
	int steps;             /* time steps to run */
	int stype;             /* ST_AOS (le_step) or ST_SOA (le_step_soa semantics and layout) */
	int receiver_row;      /* -1: none; else record vx, vy of this row every receiver_every steps */
	int receiver_every;
} le2d_problem;

typedef struct le2d_batch le2d_batch;

/* device_budget_bytes: device memory the batch may hold for states (0 = 90% of free). */
le2d_batch *le2d_batch_create(size_t device_budget_bytes);
void le2d_batch_destroy(le2d_batch *b);
/* Adds an instance; its initial state is the zero grid plus `ndisks` pressure disks
 * (disks[4k..4k+3] = cx, cy, r, s, applied in order like le_set_ball), or `init`
 * (5*nx*ny reals in the problem's layout) when not NULL.  Returns the instance id (>= 0)
 * or -LE2D_E* (e.g. -LE2D_EBUDGET when it does not fit the budget). */
int le2d_batch_add(le2d_batch *b, const le2d_problem *p, const real *init, int ndisks,
		   const real *disks);
/* Runs every instance to its step count; *device_ms (may be NULL) = device time.
 * LE2D_ETIMEOUT if a bounded wait gave up: only the instances concerned fail (their
 * le2d_batch_fields / _receivers / _diagnostics return LE2D_ETIMEOUT), the others'
 * results are valid. */
int le2d_batch_run(le2d_batch *b, int window_steps, float *device_ms);
int le2d_batch_count(const le2d_batch *b);
/* Final fields of instance `id` (5*nx*ny reals, the problem's layout). */
int le2d_batch_fields(le2d_batch *b, int id, real *out);
/* Receiver samples of instance `id`: out[s*2*nx + 0*nx + i] = vx, [... + 1*nx + i] = vy of
 * sample s (after step (s+1)*receiver_every); *nsamples = steps / receiver_every. */
int le2d_batch_receivers(le2d_batch *b, int id, real *out, int *nsamples);
int le2d_batch_diagnostics(le2d_batch *b, int id, le2d_diag_t *out);
/* Bounded dependency waits: the kernel gives up on an instance after this many ns
 * (default 2e9), skips its remaining work and le2d_batch_run returns LE2D_ETIMEOUT. */
int le2d_batch_set_wait_limit(le2d_batch *b, unsigned long long ns);
/* Batched-path autotuner: times the batched kernel on copies of a scratch problem of
 * nx x ny nodes (enough copies for ~24 M nodes) for every tile height (16 ... 256 rows) and
 * steps per work item (1, and 2 -- a producer / consumer warp pair per tile -- in the FP32
 * library), and keeps the fastest for the size class (nx, ny rounded up to powers of two).
 * Instances of a tuned class that are added to a batch afterwards use it (a server keeps the
 * default tiles, which give small solves shorter latency); with LE2D_AUTOTUNE=1
 * le2d_batch_add tunes a class on its first instance.  out (may be NULL):
 * {tile rows, steps per item}; *nu_per_s (may be NULL): the measured node-updates/s. */
int le2d_batch_autotune(int nx, int ny, int *out, double *nu_per_s);
/* Forgets every tuned size class of the batched path. */
int le2d_batch_autotune_reset(void);

/* ---- Served solves (continuous batching) --------------------------------------------
 * A background loop owns a device arena of `device_budget_bytes`.  Requests are queued
 * by le2d_server_submit (thread-safe, returns at once); the loop admits queued requests
 * while their states fit the budget (and at most `max_active` run at once), advances
 * every admitted solve in persistent launches of `window_steps` steps, and moves
 * finished ones to host-side results.  Initial states are uploaded and results read
 * back on a copy stream while the next launch runs; requests that arrive during a
 * launch join the next one.  A solve whose bounded device wait gives up fails alone
 * (LE2D_ETIMEOUT). */
#define LE2D_WANT_FIELDS 0
#define LE2D_WANT_RECEIVERS 1

typedef struct le2d_server le2d_server;

typedef struct {
	long long submitted, admitted, completed, failed;
	long long node_updates;   /* node-updates done by the device */
	long long windows;        /* persistent launches */
	double device_busy_s;     /* host time spent in launches */
	size_t arena_used, arena_capacity;
	int active, queued;
} le2d_server_stats_t;

le2d_server *le2d_server_create(size_t device_budget_bytes, int window_steps, int max_active);
/* Stops the loop; unfinished requests are dropped. */
void le2d_server_destroy(le2d_server *s);
/* Queues a solve (init/disks as le2d_batch_add; `init` is copied).  `want` =
 * LE2D_WANT_FIELDS or LE2D_WANT_RECEIVERS (needs p->receiver_row >= 0).  Returns a ticket
 * (>= 1) or -LE2D_E* (EINVAL: bad request; EBUDGET: larger than the whole budget). */
long long le2d_server_submit(le2d_server *s, const le2d_problem *p, const real *init, int ndisks,
			     const real *disks, int want);
/* 1 = finished, 0 = pending, -LE2D_E* = failed or unknown ticket. */
int le2d_server_poll(le2d_server *s, long long ticket);
/* Waits up to timeout_s (< 0: no limit): LE2D_OK, LE2D_ETIMEOUT, or the request's error. */
int le2d_server_wait(le2d_server *s, long long ticket, double timeout_s);
/* Copies a finished result: fields (5*nx*ny reals, problem layout) or receiver samples
 * ([nsamples][2][nx]); out_elems = capacity of `out`; *nsamples set for receivers. */
int le2d_server_result(le2d_server *s, long long ticket, real *out, size_t out_elems,
		       int *nsamples);
/* Host monotonic times (s) of submission, admission to the device and completion. */
int le2d_server_times(le2d_server *s, long long ticket, double *t_submit, double *t_admit,
		      double *t_done);
/* Forgets a finished ticket and its result. */
int le2d_server_release(le2d_server *s, long long ticket);
int le2d_server_stats(le2d_server *s, le2d_server_stats_t *out);
/* Host monotonic clock used by le2d_server_times (s). */
double le2d_now(void);

/* Rows [row0, row0 + nrows) of the task's current state copied to (rows_out) or from
 * (rows_in) a device buffer of the caller, laid out [field][row][nx] (5 * nrows * nx reals),
 * on the caller's CUDA stream `stream` (NULL = legacy default stream) and ordered with the
 * task's own work both ways.  For a caller that exchanges boundary rows between processes
 * itself (one process per GPU, e.g. NCCL send/recv on that stream): the rows a neighbour
 * needs go out, its rows come in as halo rows.  New surface with no counterpart in the
 * reference (whose multi-GPU variants copy rows within one process). */
int le2d_rows_out(le_task *task, int row0, int nrows, real *dev_buf, void *stream);
int le2d_rows_in(le_task *task, int row0, int nrows, const real *dev_buf, void *stream);

/* Bounds-checked build (the library under le2d_b200/lib/checked/, compiled with LE2D_CHECK):
 * every access of the state by the step kernels checks that it stays inside the buffer it
 * addresses and is skipped and counted when it does not.  Returns 1 in the checked build
 * (*count = accesses refused on the current device since the last call), 0 in the normal
 * build (*count = 0).  A stand-in for a memory checker on machines where none can run. */
int le2d_check_violations(unsigned long long *count);

/* Layout of the device state (SoA, 5 planes of n.y rows with a padded row pitch). */
int le2d_device_layout(const le_task *task, long long *pitch_elems, long long *plane_elems);

/* Bytes of device memory a task of this size holds (for admission control). */
size_t le2d_task_device_bytes(int nx, int ny);

/* Self-test of the step kernels' FP64 slope-ratio division: for i < n, fast[i] = the
 * kernels' a[i] / b[i] (a hardware reciprocal estimate, one Newton step and a Markstein
 * correction) and ieee[i] = the correctly rounded quotient, both computed on the current
 * device from host arrays.  New surface with no counterpart in the reference (whose
 * division is the compiler's). */
int le2d_selftest_ratio(const double *a, const double *b, long long n, double *fast, double *ieee);

/* Self-test of the FP64 step's limited slope ratio: for i < n, out[i] = kc * superbee(a[i] /
 * b[i]) as the FP64 kernels form it (the division above fused with the limiter; at b = +0 the
 * division's limit), computed on the current device from host arrays; it equals kc times
 * the reference's superbee (simple/le_core.c:38) of the correctly rounded quotient. */
int le2d_selftest_limiter(const double *a, const double *b, double kc, long long n, double *out);

/* ---- One grid over several devices (row slabs) ---------------------------------------
 * The reference's multi-GPU step (cuda5/cuda6 le_core.cu:374-509: one process, row slabs,
 * peer copies of the rows next to each cut).  The task's grid (its size, dt, h, material
 * and layout; not its state) is split into `nslabs` row slabs of at least 8 rows, slab i on
 * devices[i] (a device may hold several slabs).  Each slab keeps 4 copied rows beside every
 * cut, steps with the same kernels as a whole task, and refreshes those rows from its
 * neighbours after every launch, so the results are bitwise those of the whole grid.
 * Peer access between neighbouring devices is enabled where the hardware offers it. */
typedef struct le2d_slabs le2d_slabs;
le2d_slabs *le2d_slabs_create(const le_task *task, int nslabs, const int *devices);
void le2d_slabs_destroy(le2d_slabs *s);
/* Global rows [*r0, *r1) owned by slab `slab`, and its device. */
int le2d_slabs_rows(const le2d_slabs *s, int slab, int *r0, int *r1, int *device);
/* The whole state from / to a host grid in the task's layout (5*nx*ny reals). */
int le2d_slabs_upload(le2d_slabs *s, const real *src);
int le2d_slabs_download(le2d_slabs *s, real *dst);
/* nsteps steps (le_step semantics for ST_AOS grids, le_step_soa for ST_SOA); queued on
 * the slabs' streams, returns at once. */
int le2d_slabs_step_n(le2d_slabs *s, int nsteps);
int le2d_slabs_wait(le2d_slabs *s);

#ifdef __cplusplus
}
#endif

#endif /* LE2D_H */
