/*
 * Harness around the reference solver `simple/le_core.c` -- TEST INFRASTRUCTURE ONLY.
 *
 * Compiled by oracle/Makefile together with the unmodified reference source
 * (`simple/le_core.c`, its own flags `-fopenmp -O2 -fno-tree-vectorize`,
 * simple/Makefile:1-7) into oracle/_ref/libref_simple_{f,d}.so.  It exposes flat
 * C entry points so that tests and the CPU-baseline leg of bench.py can drive the
 * reference's own le_init_task / le_set_ball / le_step / le_step_soa /
 * le_save_task (simple/le_core.h:217-254) on caller-provided buffers.
 */
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "le_core.h"

int ref_real_size(void) { return (int)sizeof(real); }

/* le_init_material (simple/le_core.c:171-187); out = the 8 members in struct order. */
void ref_material(real c1, real c2, real rho, real *out)
{
    le_material m;
    le_init_material(c1, c2, rho, &m);
    memcpy(out, &m, sizeof(m));
}

static int make_task(le_task *t, int nx, int ny, real dt, real hx, real hy, real c1, real c2,
                     real rho, int stype)
{
    le_material m;
    le_vec2 h;
    le_point2 n;
    h.x = hx;
    h.y = hy;
    n.x = nx;
    n.y = ny;
    le_init_material(c1, c2, rho, &m);
    le_init_task(t, dt, h, m, n, stype);
    return t->grid ? 0 : -1;
}

/* Zero grid (le_init_task) plus balls applied in order with le_set_ball; copied to out. */
int ref_initial_state(int nx, int ny, real hx, real hy, int stype, int nballs, const real *cx,
                      const real *cy, const real *r, const real *s, real *out)
{
    le_task t;
    int b;
    if (make_task(&t, nx, ny, 0, hx, hy, 1, 0.5, 1, stype))
        return -1;
    for (b = 0; b < nballs; b++) {
        le_vec2 c;
        c.x = cx[b];
        c.y = cy[b];
        le_set_ball(&t, c, r[b], s[b]);
    }
    memcpy(out, t.grid, sizeof(le_node) * (size_t)nx * ny);
    le_free_task(&t);
    return 0;
}

/* Runs `steps` reference steps on grid_inout (layout given by stype) with `threads`
 * OpenMP threads; returns the wall time of the step loop in seconds (<0 on error). */
double ref_run(int nx, int ny, real dt, real hx, real hy, real c1, real c2, real rho, int stype,
               real *grid_inout, int steps, int threads)
{
    le_task t;
    int s;
    double t0, t1;
    if (make_task(&t, nx, ny, dt, hx, hy, c1, c2, rho, stype))
        return -1.0;
    memcpy(t.grid, grid_inout, sizeof(le_node) * (size_t)nx * ny);
    if (threads > 0)
        omp_set_num_threads(threads);
    t0 = omp_get_wtime();
    for (s = 0; s < steps; s++) {
        if (stype == ST_AOS)
            le_step(&t);
        else
            le_step_soa(&t);
    }
    t1 = omp_get_wtime();
    memcpy(grid_inout, t.grid, sizeof(le_node) * (size_t)nx * ny);
    le_free_task(&t);
    return t1 - t0;
}

/* le_save_task on a copy of `grid`. */
int ref_save(int nx, int ny, real hx, real hy, int stype, const real *grid, const char *path)
{
    le_task t;
    int rc;
    if (make_task(&t, nx, ny, 0, hx, hy, 1, 0.5, 1, stype))
        return -1;
    memcpy(t.grid, grid, sizeof(le_node) * (size_t)nx * ny);
    rc = le_save_task(&t, path);
    le_free_task(&t);
    return rc;
}
