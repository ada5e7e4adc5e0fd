/*
 * Harness around the reference's pthread solver `pthread/le_core.c` -- TEST
 * INFRASTRUCTURE ONLY, used as a timed CPU speed baseline (never as an oracle:
 * its rearranged tvd2, pthread/le_core.c:26-45, is not numerically equal to
 * simple/).  Mirrors the flow of pthread/main.c:22-84: init, one thread per slab
 * running the reference's le_step thread body, join.
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "le_core.h"

extern pthread_barrier_t b; /* defined in pthread/le_core.c:24 */

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int ref_pthread_real_size(void) { return (int)sizeof(real); }

/* grid_inout: AOS state (may be NULL for an all-zero start).  Returns seconds for
 * thread create .. join, or <0 on error.  threads must satisfy ny / threads >= 4. */
double ref_pthread_run(int nx, int ny, real dt, real hx, real hy, real c1, real c2, real rho,
                       real *grid_inout, int steps, int threads)
{
    le_task task;
    le_material mat;
    le_vec2 h;
    le_point2 n;
    pthread_t *tid;
    st_pthread *data;
    int ti;
    double t0, t1;
    if (threads < 1 || ny / threads < 4)
        return -1.0;
    h.x = hx;
    h.y = hy;
    n.x = nx;
    n.y = ny;
    le_init_material(c1, c2, rho, &mat);
    task.max_threads = threads;
    task.steps = steps;
    le_init_task(&task, dt, h, mat, n);
    /* pthread/le_core.c:90 zeroes only part of the grid; set every byte here. */
    if (grid_inout)
        memcpy(task.grid, grid_inout, sizeof(real) * NODE_SIZE * (size_t)nx * ny);
    else
        memset(task.grid, 0, sizeof(real) * NODE_SIZE * (size_t)nx * ny);
    tid = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    data = (st_pthread *)malloc(sizeof(st_pthread) * threads);
    pthread_barrier_init(&b, NULL, threads);
    t0 = now_s();
    for (ti = 0; ti < threads; ti++) {
        data[ti].task = &task;
        data[ti].thread_num = ti;
        if (pthread_create(&tid[ti], NULL, le_step, &data[ti]))
            return -2.0;
    }
    for (ti = 0; ti < threads; ti++)
        pthread_join(tid[ti], NULL);
    t1 = now_s();
    pthread_barrier_destroy(&b);
    if (grid_inout)
        memcpy(grid_inout, task.grid, sizeof(real) * NODE_SIZE * (size_t)nx * ny);
    le_free_task(&task);
    free(tid);
    free(data);
    return t1 - t0;
}
