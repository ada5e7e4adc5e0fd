/*
 * Harness around the reference's two-buffer schedule `tiling/le_core.c` -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * Compiled by oracle/Makefile together with the unmodified reference source (its own flags,
 * tiling/Makefile: -O2) into oracle/_ref/libref_tiling_{f,d}.so.  It drives the reference's
 * le_step_all2 (tiling/le_core.c:670-708): Jacobi steps between two buffers with a zero ring
 * of two nodes around the grid (not the clamped ends of simple/), and increments associated
 * as (v + d1) + d2 (tiling/le_core.c:258-285) where simple/ adds v + (d1 + d2).  Away from the
 * edges (2 nodes per step) it computes simple/'s step with other roundings: an independent
 * schedule to check the library's temporal blocking against.
 */
#include <string.h>
#include "le_core.h"

/* Defined in tiling/le_core.c:670-708, not declared in its header. */
void le_step_all2(le_task *t, int steps);

int ref_tiling_real_size(void) { return (int)sizeof(real); }

/* `steps` time steps of the AoS grid (nx * ny nodes, in place) by le_step_all2. */
int ref_tiling_run(int nx, int ny, real dt, real hx, real hy, real c1, real c2, real rho,
                   real *grid, int steps)
{
    le_material m;
    le_vec2 h;
    le_point2 n;
    le_task t;
    le_node *g, *in = (le_node *)grid;
    size_t padded = sizeof(le_node) * (size_t)(nx + 4) * (size_t)(ny + 4);
    int i, j;
    h.x = hx;
    h.y = hy;
    n.x = nx;
    n.y = ny;
    le_init_material(c1, c2, rho, &m);
    le_init_task(&t, dt, h, m, n, ST_AOS);
    if (!t.grid || !t.grid2)
        return -1;
    /* le_init_task clears only nx * ny nodes of each padded buffer (tiling/le_core.c:128-129);
     * the zero ring the schedule reads needs all of them cleared */
    memset(t.grid, 0, padded);
    memset(t.grid2, 0, padded);
    g = (le_node *)t.grid;
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++)
            g[(i + 2) + (j + 2) * (nx + 4)] = in[i + j * nx];
    le_step_all2(&t, steps);
    for (j = 0; j < ny; j++)
        for (i = 0; i < nx; i++)
            in[i + j * nx] = g[(i + 2) + (j + 2) * (nx + 4)];
    le_free_task(&t);
    return 0;
}
