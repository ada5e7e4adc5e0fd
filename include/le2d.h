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

/* Step kernels: FUSED = one kernel per step (x- and y-sweep fused per strip);
 * SPLIT = the plain scheme, one kernel per sweep. */
#define LE2D_METHOD_FUSED 0
#define LE2D_METHOD_SPLIT 1
int le2d_set_method(le_task *task, int method);

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

/* Layout of the device state (SoA, 5 planes of n.y rows with a padded row pitch). */
int le2d_device_layout(const le_task *task, long long *pitch_elems, long long *plane_elems);

/* Bytes of device memory a task of this size holds (for admission control). */
size_t le2d_task_device_bytes(int nx, int ny);

#ifdef __cplusplus
}
#endif

#endif /* LE2D_H */
