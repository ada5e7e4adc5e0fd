/*
 * le_core.h -- le2d task API, B200 implementation (lible2d_f.so / lible2d_d.so).
 *
 * Drop-in replacement for the reference task API in le2d `simple/le_core.h`:
 * the same types with byte-identical layouts, the same function names,
 * signatures and argument meaning, so a C host written against the reference
 * (e.g. its `simple/main.c`) compiles and links against this library unchanged.
 * Precision is a compile-time type exactly as in the reference: define
 * USE_DOUBLE and link lible2d_d.so for double, otherwise link lible2d_f.so.
 *
 * The state lives on the GPU between calls; `task->grid` is the host copy and is
 * brought up to date by le_save_task, le2d_sync_host (le2d.h) and le_free_task.
 * Extensions (explicit sync, error query, multi-step calls, diagnostics, batched
 * and served solves) are declared in le2d.h.
 */
#ifndef LE_CORE_H
#define LE_CORE_H

#include <sys/time.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Wall-clock and cycle-counter helpers the reference driver uses
 * (simple/le_core.h:13-26; simple/main.c:54-55). */
static __inline__ unsigned long getCC(void)
{
#if defined(__x86_64__) || defined(__i386__)
	unsigned lo, hi;
	__asm__ __volatile__("rdtsc" : "=a"(lo), "=d"(hi));
	return ((unsigned long)lo) | (((unsigned long)hi) << 32);
#else
	return 0;
#endif
}

static __inline__ double timer(void)
{
	struct timeval tv;
	gettimeofday(&tv, 0);
	return tv.tv_sec + 1e-6 * tv.tv_usec;
}

/* Storage types (simple/le_core.h:34-35). */
#define ST_SOA 0
#define ST_AOS 1

/* Real type (simple/le_core.h:37-61). */
#ifdef USE_DOUBLE
typedef double real;
#else
typedef float real;
#endif

typedef int int_t;                                          /* simple/le_core.h:131 */
typedef struct { real x, y; } le_vec2;                      /* simple/le_core.h:134-136 */
typedef struct { real xx, xy, yy; } le_smatrix2;            /* simple/le_core.h:143-145 */
typedef struct { int_t x, y; } le_point2;                   /* simple/le_core.h:148-150 */
typedef struct { le_vec2 v; le_smatrix2 s; } le_node;       /* simple/le_core.h:156-159 */
typedef struct { real w1, w2, w3, w4; } le_w;               /* simple/le_core.h:164-166 */

/* Material: P speed c1, S speed c2, density rho, and cached products
 * (simple/le_core.h:175-186). */
typedef struct {
	real c1, c2, rho;
	real irhoc1; /* 1 / (c1 rho) */
	real irhoc2; /* 1 / (c2 rho) */
	real rhoc1;  /* c1 rho */
	real rhoc2;  /* c2 rho */
	real rhoc3;  /* rho c1 la / (la + 2 mu) */
} le_material;

/* Task (simple/le_core.h:191-212). */
typedef struct {
	real dt;
	le_vec2 h;
	le_point2 n;
	le_material mat;
	int stype;
	real *grid;
} le_task;

/* simple/le_core.h:217 -- fills m, including the cached products. */
void le_init_material(const real c1, const real c2, const real rho, le_material *m);

/* simple/le_core.h:220 -- allocates and zeroes task->grid (5*n.x*n.y reals, host, page-locked
 * when possible) and the task's device state.  n.x, n.y >= 3. */
void le_init_task(le_task *task, const real dt, const le_vec2 h, const le_material mat,
		  const le_point2 n, const int stype);

/* simple/le_core.h:223 -- releases the host grid and the device state. */
void le_free_task(le_task *task);

/* simple/le_core.h:228 -- sets sxx = syy = s at every node (h.x*i, h.y*j) strictly inside the
 * disk of radius r around c (applied to the current state, host or device). */
void le_set_ball(le_task *t, const le_vec2 c, const real r, const real s);

/* simple/le_core.h:237 -- legacy VTK (|v| as big-endian float32).  0 = ok, 1 = error. */
int le_save_task(le_task *task, const char *file);

/* simple/le_core.h:242 -- one time step (x-sweep then y-sweep) of an ST_AOS task. */
void le_step(le_task *task);

/* simple/le_core.h:254 -- one time step of an ST_SOA task.  Reproduces the reference SoA
 * step exactly, including its far end of the y-sweep: past the last row its stencil sees
 * rows n.y-5 and n.y-4 (clamped at 0) instead of copies of row n.y-1
 * (simple/le_core.c:329-349), so it equals le_step until waves reach that edge. */
void le_step_soa(le_task *task);

#ifdef __cplusplus
}
#endif

#endif /* LE_CORE_H */
