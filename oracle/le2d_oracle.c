/*
 * le2d CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference solver's time step (le2d `simple/`),
 * used by the test-suite, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg as the checker.  Nothing in the product library links or calls
 * this file.
 *
 * Parity pin: every function here follows the operation order and the C type
 * promotions of `simple/le_core.c`, so that the float build and the double
 * build reproduce the reference's own float and double builds bit for bit.
 * tests/test_oracle.py checks that against the golden fixtures made by running
 * the reference itself (tests/golden/make_golden.py, oracle/Makefile).
 *
 * Compiled twice (see oracle/Makefile): default real_t = float,
 * -DORACLE_DOUBLE gives real_t = double.  -ffp-contract=off keeps the compiler
 * from fusing multiply-adds that the reference build (x86-64 baseline, no FMA)
 * does not fuse.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>

#ifdef ORACLE_DOUBLE
typedef double real_t;
#else
typedef float real_t;
#endif

/* Field order inside a node: simple/le_core.h:156-159 (le_node = {v.x, v.y, s.xx, s.xy, s.yy})
 * and simple/le_core.c:17-21 (SoA planes in the same order). */
enum { F_VX = 0, F_VY = 1, F_SXX = 2, F_SXY = 3, F_SYY = 4, NFIELD = 5 };

/* Storage types: simple/le_core.h:34-35. */
enum { STORE_SOA = 0, STORE_AOS = 1 };

/* Material with cached products, same member order as le_material (simple/le_core.h:175-186). */
typedef struct {
    real_t c1, c2, rho;
    real_t irhoc1, irhoc2, rhoc1, rhoc2, rhoc3;
} o_material;

/* simple/le_core.c:171-187.  The double literals promote the divisions and the
 * `2.0 * mu` terms to double before the result is stored back as real_t. */
void oracle_material(real_t c1, real_t c2, real_t rho, o_material *m)
{
    m->c1 = c1;
    m->c2 = c2;
    m->rho = rho;
    m->irhoc1 = 1.0 / (c1 * rho);
    m->irhoc2 = 1.0 / (c2 * rho);
    m->rhoc1 = c1 * rho;
    m->rhoc2 = c2 * rho;
    {
        real_t mu = rho * c2 * c2;
        real_t la = rho * c1 * c1 - 2.0 * mu;
        m->rhoc3 = rho * c1 * la / (la + 2.0 * mu);
    }
}

/* TVD2_EPS: simple/le_core.c:29 (a double literal, so `x += EPS` rounds once from double). */
#define O_EPS 1e-6

/* le_min / le_max / le_max3: simple/le_core.c:31-33 (real_t parameters, so a double
 * argument such as `2.0 * r` is rounded to real_t at the call). */
static inline real_t o_min(real_t a, real_t b) { return a > b ? b : a; }
static inline real_t o_max(real_t a, real_t b) { return a > b ? a : b; }

/* Superbee limiter: simple/le_core.c:38 (max3(0, min(1, 2r), min(2, r))). */
static inline real_t o_superbee(real_t r)
{
    return o_max(0.0, o_max(o_min(1.0, 2.0 * r), o_min(2.0, r)));
}

/* Second-order TVD update of one invariant: simple/le_core.c:48-69.
 * Stencil (up2, up1, u, dn1) is ordered along the characteristic's direction of travel.
 * The limited fluxes are formed in double (`phi / 2.0 * (1.0 - c) * diff`) and
 * rounded to real_t when stored, as in the reference. */
static inline real_t o_tvd2(real_t c, real_t up2, real_t up1, real_t u, real_t dn1)
{
    real_t num = u - up1;
    real_t den = dn1 - u;
    num += O_EPS;
    den += O_EPS;
    const real_t r_here = num / den;
    num = up1 - up2;
    den = u - up1;
    num += O_EPS;
    den += O_EPS;
    const real_t r_prev = num / den;
    const real_t flux_out = u + o_superbee(r_here) / 2.0 * (1.0 - c) * (dn1 - u);
    const real_t flux_in = up1 + o_superbee(r_prev) / 2.0 * (1.0 - c) * (u - up1);
    return u - c * (flux_out - flux_in);
}

/*
 * One directional sweep of one grid line (a row for axis 0, a column for axis 1).
 *
 * Invariants along axis a (simple/le_core.c:192-218): with vn/vt the normal and
 * tangential velocity and sn the normal stress,
 *     w1 = vn - sn*irhoc1, w2 = vn + sn*irhoc1, w3 = vt - sxy*irhoc2, w4 = vt + sxy*irhoc2.
 * All invariants of the line are formed before any node is updated (the
 * reference's rolling window reads node i+3 before writing node i, which is the
 * same Jacobi order), with the index clamped to [0, n-1] at both ends
 * (simple/le_core.c:482-486 and :496).  w1/w3 move toward +a (stencil i-2..i+1),
 * w2/w4 toward -a (mirrored stencil): reconstruct, simple/le_core.c:251-257.
 * The update is inc_x / inc_y, simple/le_core.c:221-249.
 */
static void o_sweep_line(real_t *g, ptrdiff_t node_stride, ptrdiff_t field_stride, int n,
                         int axis, const o_material *m, real_t k1, real_t k2, real_t *w,
                         int far_end_rotated)
{
    const int f_vn = axis == 0 ? F_VX : F_VY;
    const int f_vt = axis == 0 ? F_VY : F_VX;
    const int f_sn = axis == 0 ? F_SXX : F_SYY;
    const int f_so = axis == 0 ? F_SYY : F_SXX;
    int i;
    /* w[(i + 2) * 4 + k] holds invariant k+1 of node clamp(i) for i in [-2, n+1]. */
    for (i = 0; i < n; i++) {
        const real_t *nd = g + (ptrdiff_t)i * node_stride;
        const real_t n00 = nd[f_sn * field_stride] * m->irhoc1;
        const real_t n01 = nd[F_SXY * field_stride] * m->irhoc2;
        real_t *wi = w + (ptrdiff_t)(i + 2) * 4;
        wi[0] = nd[f_vn * field_stride] - n00;
        wi[1] = nd[f_vn * field_stride] + n00;
        wi[2] = nd[f_vt * field_stride] - n01;
        wi[3] = nd[f_vt * field_stride] + n01;
    }
    for (i = 0; i < 4; i++) {
        w[0 * 4 + i] = w[1 * 4 + i] = w[2 * 4 + i];
        if (!far_end_rotated) {
            w[(n + 3) * 4 + i] = w[(n + 2) * 4 + i] = w[(n + 1) * 4 + i];
        } else {
            /* le_soa_step_y (simple/le_core.c:329-349) rotates five row buffers and stops
             * refreshing them at j = n-3, so past the last row its window sees the rows
             * n-5 and n-4 (index clamped at 0) instead of copies of row n-1. */
            w[(n + 2) * 4 + i] = w[((n - 5 > 0 ? n - 5 : 0) + 2) * 4 + i];
            w[(n + 3) * 4 + i] = w[((n - 4 > 0 ? n - 4 : 0) + 2) * 4 + i];
        }
    }
    for (i = 0; i < n; i++) {
        const real_t *a2 = w + (ptrdiff_t)(i + 0) * 4; /* node i-2 */
        const real_t *a1 = w + (ptrdiff_t)(i + 1) * 4; /* node i-1 */
        const real_t *c0 = w + (ptrdiff_t)(i + 2) * 4; /* node i   */
        const real_t *b1 = w + (ptrdiff_t)(i + 3) * 4; /* node i+1 */
        const real_t *b2 = w + (ptrdiff_t)(i + 4) * 4; /* node i+2 */
        real_t d1 = o_tvd2(k1, a2[0], a1[0], c0[0], b1[0]) - c0[0];
        real_t d2 = o_tvd2(k1, b2[1], b1[1], c0[1], a1[1]) - c0[1];
        real_t d3 = o_tvd2(k2, a2[2], a1[2], c0[2], b1[2]) - c0[2];
        real_t d4 = o_tvd2(k2, b2[3], b1[3], c0[3], a1[3]) - c0[3];
        d1 *= 0.5;
        d2 *= 0.5;
        d3 *= 0.5;
        d4 *= 0.5;
        {
            real_t *nd = g + (ptrdiff_t)i * node_stride;
            nd[f_vn * field_stride] += d1 + d2;
            nd[f_vt * field_stride] += d3 + d4;
            nd[f_sn * field_stride] += (d2 - d1) * m->rhoc1;
            nd[f_so * field_stride] += (d2 - d1) * m->rhoc3;
            nd[F_SXY * field_stride] += m->rhoc2 * (d4 - d3);
        }
    }
}

/*
 * One time step: x-sweep of every row, then y-sweep of every column
 * (dimension splitting, simple/le_core.c:605-620).  For SoA storage this is
 * le_step_soa (simple/le_core.c:623-627), which matches le_step except at the far
 * end of the y-sweep (see o_sweep_line).  Courant numbers k = dt * c / h in real_t
 * (simple/le_core.c:468-469 and :511-512).  Returns 0, or -1 on bad arguments
 * (the reference asserts, simple/le_core.c:437 and :261).
 */
int oracle_step(real_t *grid, int nx, int ny, real_t dt, real_t hx, real_t hy,
                const o_material *m, int stype)
{
    int i, j;
    real_t *w;
    const ptrdiff_t plane = (ptrdiff_t)nx * ny;
    const ptrdiff_t fstride = stype == STORE_AOS ? 1 : plane;
    const ptrdiff_t xstride = stype == STORE_AOS ? NFIELD : 1;
    if (nx < 3 || ny < 3 || (stype != STORE_AOS && stype != STORE_SOA))
        return -1;
    w = (real_t *)malloc(sizeof(real_t) * 4 * (size_t)((nx > ny ? nx : ny) + 4));
    if (!w)
        return -1;
    {
        const real_t k1 = dt * m->c1 / hx;
        const real_t k2 = dt * m->c2 / hx;
        for (j = 0; j < ny; j++)
            o_sweep_line(grid + (ptrdiff_t)j * nx * xstride, xstride, fstride, nx, 0, m, k1, k2, w, 0);
    }
    {
        const real_t k1 = dt * m->c1 / hy;
        const real_t k2 = dt * m->c2 / hy;
        for (i = 0; i < nx; i++)
            o_sweep_line(grid + (ptrdiff_t)i * xstride, (ptrdiff_t)nx * xstride, fstride, ny, 1, m, k1, k2, w,
                         stype == STORE_SOA);
    }
    free(w);
    return 0;
}

int oracle_run(real_t *grid, int nx, int ny, real_t dt, real_t hx, real_t hy,
               const o_material *m, int stype, int steps)
{
    int s;
    for (s = 0; s < steps; s++)
        if (oracle_step(grid, nx, ny, dt, hx, hy, m, stype))
            return -1;
    return 0;
}

/* Pressure disk: simple/le_core.c:71-94.  Node (i, j) sits at (hx*i, hy*j) in real_t;
 * the distance is sqrt() of a real_t sum, compared in double with `r`. Sets (not adds)
 * sxx = syy = s inside the open disk. */
int oracle_set_ball(real_t *grid, int nx, int ny, real_t hx, real_t hy, int stype,
                    real_t cx, real_t cy, real_t r, real_t s)
{
    int i, j;
    const ptrdiff_t plane = (ptrdiff_t)nx * ny;
    if (stype != STORE_AOS && stype != STORE_SOA)
        return -1;
    for (i = 0; i < nx; i++) {
        for (j = 0; j < ny; j++) {
            const real_t px = hx * i;
            const real_t py = hy * j;
            const real_t dx = px - cx;
            const real_t dy = py - cy;
            if (sqrt(dx * dx + dy * dy) < r) {
                const ptrdiff_t node = i + (ptrdiff_t)j * nx;
                if (stype == STORE_AOS) {
                    grid[node * NFIELD + F_SXX] = s;
                    grid[node * NFIELD + F_SYY] = s;
                } else {
                    grid[F_SXX * plane + node] = s;
                    grid[F_SYY * plane + node] = s;
                }
            }
        }
    }
    return 0;
}

/* Legacy VTK writer: simple/le_core.c:130-169 with write_float :99-111.
 * Header text, then |v| = sqrt(vx^2 + vy^2) as big-endian float32, j outer, i inner. */
int oracle_save_vtk(const real_t *grid, int nx, int ny, real_t hx, real_t hy, int stype,
                    const char *path)
{
    int i, j;
    const ptrdiff_t plane = (ptrdiff_t)nx * ny;
    FILE *fp = fopen(path, "w");
    if (!fp)
        return 1;
    fprintf(fp, "# vtk DataFile Version 3.0\n");
    fprintf(fp, "Created by le_save_task\n");
    fprintf(fp, "BINARY\n");
    fprintf(fp, "DATASET STRUCTURED_POINTS\n");
    fprintf(fp, "DIMENSIONS %d %d 1\n", nx, ny);
    fprintf(fp, "SPACING %f %f 0.0\n", hx, hy);
    fprintf(fp, "ORIGIN 0.0 0.0 0.0\n");
    fprintf(fp, "POINT_DATA %d\n", nx * ny);
    fprintf(fp, "SCALARS v float 1\n");
    fprintf(fp, "LOOKUP_TABLE v_table\n");
    for (j = 0; j < ny; j++) {
        for (i = 0; i < nx; i++) {
            const ptrdiff_t node = i + (ptrdiff_t)j * nx;
            real_t vx, vy;
            float v;
            unsigned char le[4], be[4];
            if (stype == STORE_AOS) {
                vx = grid[node * NFIELD + F_VX];
                vy = grid[node * NFIELD + F_VY];
            } else {
                vx = grid[F_VX * plane + node];
                vy = grid[F_VY * plane + node];
            }
            v = sqrt(vx * vx + vy * vy);
            memcpy(le, &v, 4);
            be[0] = le[3];
            be[1] = le[2];
            be[2] = le[1];
            be[3] = le[0];
            fwrite(be, 1, 4, fp);
        }
    }
    fclose(fp);
    return 0;
}

/*
 * FP64 diagnostics of one state (not in the reference; defines what the GPU
 * diagnostic kernel must return).  Elastic energy of the 2D velocity-stress
 * system that the scheme integrates (rho dv/dt = div(sigma), isotropic,
 * lambda = rho*c1^2 - 2*mu, mu = rho*c2^2):
 *   e = rho/2 |v|^2 + [(la+2mu)(sxx^2+syy^2) - 2 la sxx syy] / (8 mu (la+mu)) + sxy^2 / (2 mu)
 * summed over nodes and multiplied by hx*hy.  out[0] = energy,
 * out[1..5] = sum of squares per field, out[6..10] = max |field|.
 */
int oracle_diag(const real_t *grid, int nx, int ny, double hx, double hy, double c1, double c2,
                double rho, int stype, double *out)
{
    const ptrdiff_t plane = (ptrdiff_t)nx * ny;
    const double mu = rho * c2 * c2;
    const double la = rho * c1 * c1 - 2.0 * mu;
    const double a_nn = (la + 2.0 * mu) / (8.0 * mu * (la + mu));
    const double a_xy = -2.0 * la / (8.0 * mu * (la + mu));
    const double a_s = 1.0 / (2.0 * mu);
    double e = 0.0;
    ptrdiff_t q;
    int f;
    for (f = 0; f < 11; f++)
        out[f] = 0.0;
    for (q = 0; q < plane; q++) {
        double v[NFIELD];
        for (f = 0; f < NFIELD; f++) {
            v[f] = stype == STORE_AOS ? grid[q * NFIELD + f] : grid[f * plane + q];
            out[1 + f] += v[f] * v[f];
            if (fabs(v[f]) > out[6 + f])
                out[6 + f] = fabs(v[f]);
        }
        e += 0.5 * rho * (v[F_VX] * v[F_VX] + v[F_VY] * v[F_VY]) +
             a_nn * (v[F_SXX] * v[F_SXX] + v[F_SYY] * v[F_SYY]) + a_xy * v[F_SXX] * v[F_SYY] +
             a_s * v[F_SXY] * v[F_SXY];
    }
    out[0] = e * hx * hy;
    return 0;
}

int oracle_real_size(void) { return (int)sizeof(real_t); }
