/*
 * er_oracle_cells.c -- the FP64 pair sum of er_oracle.c over a cell list.
 *
 * TEST INFRASTRUCTURE ONLY (see er_oracle.h). The reference's sum
 * (src/computegridsheet.h:54-92, src/doHenry.h:70-98) visits every image of
 * every atom; this restatement visits only the Cartesian cells within the
 * cutoff of a point, so a 1e7-insertion Henry run or a full grid of a large
 * framework finishes in seconds instead of minutes. Per term it evaluates
 * exactly the reference's expressions, in its order, with no contraction:
 *   image  x_w = T (x_f + i, y_f + j, z_f + k)       (src/computegridsheet.h:58-76)
 *   r^2    = dx*dx + dy*dy + dz*dz, clamped to min_r^2 (:77-78)
 *   term   = ((4 eps) s6) (s6 - 1), s2 = sig2 / r^2, s6 = s2 s2 s2, if r^2 < rc^2 (:79-82)
 * so the set of summed terms and every term's value equal the reference's;
 * only the order of the additions differs (cell by cell instead of image by
 * image), which moves a sum by a few ulps of sum |term|. tests/
 * test_oracle_pin.py pins it against the image-loop restatement. Cells are
 * visited with a 1e-6 A margin beyond the cutoff, far above the rounding of
 * the cell index, so no in-cutoff image is skipped. Atoms with eps == 0 or
 * sig2 == 0 are left out: their terms are exactly zero.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "er_oracle.h"

typedef struct {
    double x, y, z;  /* image position, the reference's expression */
    double c4, s2;   /* 4 eps (rounded as the reference's first product), sig2 */
} cimg_t;

typedef struct {
    cimg_t* img;     /* cell-sorted */
    int* start;      /* ncell + 1 */
    int nc[3];
    double lo[3], h;
    const double* t;
    double rc2, r2min;
} cells_t;

static inline void f2c(const double t[9], double xf, double yf, double zf, double* x, double* y,
                       double* z) {
    *x = t[0] * xf + t[1] * yf + t[2] * zf;
    *y = t[3] * xf + t[4] * yf + t[5] * zf;
    *z = t[6] * xf + t[7] * yf + t[8] * zf;
}

static int cell_coord(double v, double lo, double h, int n) {
    int c = (int)floor((v - lo) / h);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

static int cells_build(cells_t* C, const or_particle* atoms, int n_atoms, const double t[9],
                       const int rep[3], double rc2, double min_r) {
    memset(C, 0, sizeof(*C));
    C->t = t;
    C->rc2 = rc2;
    C->r2min = min_r * min_r;
    const int64_t per = (int64_t)(2 * rep[0] + 1) * (2 * rep[1] + 1) * (2 * rep[2] + 1);
    int64_t n = 0;
    for (int a = 0; a < n_atoms; a++)
        if (atoms[a].eps_with_adsorbate != 0.0 && atoms[a].sig_with_adsorbate_squared != 0.0)
            n += per;
    cimg_t* tmp = (cimg_t*)malloc(sizeof(cimg_t) * (size_t)(n > 0 ? n : 1));
    if (!tmp) return -1;
    int64_t q = 0;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = -rep[0]; i <= rep[0]; i++)
        for (int j = -rep[1]; j <= rep[1]; j++)
            for (int k = -rep[2]; k <= rep[2]; k++)
                for (int a = 0; a < n_atoms; a++) {
                    if (atoms[a].eps_with_adsorbate == 0.0 ||
                        atoms[a].sig_with_adsorbate_squared == 0.0)
                        continue;
                    cimg_t* m = &tmp[q++];
                    f2c(t, atoms[a].x_f + 1.0 * i, atoms[a].y_f + 1.0 * j, atoms[a].z_f + 1.0 * k,
                        &m->x, &m->y, &m->z);
                    m->c4 = 4.0 * atoms[a].eps_with_adsorbate;
                    m->s2 = atoms[a].sig_with_adsorbate_squared;
                    const double v[3] = {m->x, m->y, m->z};
                    for (int d = 0; d < 3; d++) {
                        if (v[d] < lo[d]) lo[d] = v[d];
                        if (v[d] > hi[d]) hi[d] = v[d];
                    }
                }
    const double rc = sqrt(rc2);
    C->h = rc > 1.0 ? rc / 3.0 : 1.0;
    int64_t ncell = 1;
    for (int d = 0; d < 3; d++) {
        if (n == 0) { lo[d] = 0.0; hi[d] = 0.0; }
        C->lo[d] = lo[d];
        C->nc[d] = (int)floor((hi[d] - lo[d]) / C->h) + 1;
        if (C->nc[d] < 1) C->nc[d] = 1;
        ncell *= C->nc[d];
    }
    C->start = (int*)calloc((size_t)ncell + 1, sizeof(int));
    C->img = (cimg_t*)malloc(sizeof(cimg_t) * (size_t)(n > 0 ? n : 1));
    int* cell = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!C->start || !C->img || !cell) {
        free(tmp); free(cell);
        return -1;
    }
    for (int64_t p = 0; p < n; p++) {
        const int cx = cell_coord(tmp[p].x, C->lo[0], C->h, C->nc[0]);
        const int cy = cell_coord(tmp[p].y, C->lo[1], C->h, C->nc[1]);
        const int cz = cell_coord(tmp[p].z, C->lo[2], C->h, C->nc[2]);
        cell[p] = (cz * C->nc[1] + cy) * C->nc[0] + cx;
        C->start[cell[p] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) C->start[c + 1] += C->start[c];
    int* fill = (int*)malloc(sizeof(int) * (size_t)ncell);
    memcpy(fill, C->start, sizeof(int) * (size_t)ncell);
    for (int64_t p = 0; p < n; p++) C->img[fill[cell[p]]++] = tmp[p];
    free(fill);
    free(cell);
    free(tmp);
    return 0;
}

static void cells_free(cells_t* C) {
    free(C->img);
    free(C->start);
}

/* Energy, sum |term| and in-cutoff count at the fractional point f. */
static void cells_point(const cells_t* C, double xf, double yf, double zf, double* e_out,
                        double* abs_out, int64_t* n_out) {
    double x, y, z;
    f2c(C->t, xf, yf, zf, &x, &y, &z);
    const double R = sqrt(C->rc2) + 1e-6;
    const double p[3] = {x, y, z};
    int c0[3], c1[3];
    for (int d = 0; d < 3; d++) {
        c0[d] = cell_coord(p[d] - R, C->lo[d], C->h, C->nc[d]);
        c1[d] = cell_coord(p[d] + R, C->lo[d], C->h, C->nc[d]);
    }
    double energy = 0.0, sabs = 0.0;
    int64_t n = 0;
    for (int cz = c0[2]; cz <= c1[2]; cz++)
        for (int cy = c0[1]; cy <= c1[1]; cy++) {
            const int row = (cz * C->nc[1] + cy) * C->nc[0];
            const int b = C->start[row + c0[0]], e = C->start[row + c1[0] + 1];
            for (int q = b; q < e; q++) {
                const cimg_t* m = &C->img[q];
                double dx = x - m->x, dy = y - m->y, dz = z - m->z;
                double r2 = dx * dx + dy * dy + dz * dz;
                r2 = (r2 > C->r2min) ? r2 : C->r2min;
                if (r2 < C->rc2) {
                    double s2 = m->s2 / r2;
                    double s6 = s2 * s2 * s2;
                    double term = m->c4 * s6 * (s6 - 1.0);
                    energy += term;
                    sabs += fabs(term);
                    n++;
                }
            }
        }
    if (e_out) *e_out = energy;
    if (abs_out) *abs_out = sabs;
    if (n_out) *n_out = n;
}

static int nthreads(int n_threads, int64_t work) {
    long n = n_threads > 0 ? n_threads : sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1) n = 1;
    if ((int64_t)n > work) n = work > 0 ? (int)work : 1;
    return (int)n;
}

typedef struct {
    const cells_t* C;
    const double* pts;
    int64_t n;
    double *e, *sabs, *cnt;
    int tid, nth;
} cjob_t;

static void* points_fn(void* arg) {
    cjob_t* j = (cjob_t*)arg;
    for (int64_t p = j->tid; p < j->n; p += j->nth) {
        double e, s;
        int64_t c;
        cells_point(j->C, j->pts[3 * p], j->pts[3 * p + 1], j->pts[3 * p + 2], &e, &s, &c);
        if (j->e) j->e[p] = e;
        if (j->sabs) j->sabs[p] = s;
        if (j->cnt) j->cnt[p] = (double)c;
    }
    return NULL;
}

int oracle_points_cells(const or_particle* atoms, int n_atoms, const double t[9],
                        const int rep[3], double rc2, double min_r, const double* pts,
                        int64_t n_pts, double* energy, double* sum_abs, double* n_terms,
                        int n_threads) {
    cells_t C;
    if (cells_build(&C, atoms, n_atoms, t, rep, rc2, min_r)) return -1;
    const int nth = nthreads(n_threads, n_pts);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nth);
    cjob_t* jobs = (cjob_t*)calloc((size_t)nth, sizeof(cjob_t));
    for (int k = 0; k < nth; k++) {
        jobs[k].C = &C; jobs[k].pts = pts; jobs[k].n = n_pts;
        jobs[k].e = energy; jobs[k].sabs = sum_abs; jobs[k].cnt = n_terms;
        jobs[k].tid = k; jobs[k].nth = nth;
        pthread_create(&th[k], NULL, points_fn, &jobs[k]);
    }
    for (int k = 0; k < nth; k++) pthread_join(th[k], NULL);
    free(th);
    free(jobs);
    cells_free(&C);
    return 0;
}

/* Grid axes i/(N-1) (src/writegrid.cu:122-127), layout k + j nz + i ny nz. */
typedef struct {
    const cells_t* C;
    int nx, ny, nz;
    double *e, *sabs;
    int tid, nth;
} gjob_t;

static void* grid_fn(void* arg) {
    gjob_t* j = (gjob_t*)arg;
    for (int i = j->tid; i < j->nx; i += j->nth) {
        const double xf = 1.0 * i / (j->nx - 1);
        for (int jj = 0; jj < j->ny; jj++) {
            const double yf = 1.0 * jj / (j->ny - 1);
            for (int k = 0; k < j->nz; k++) {
                const double zf = 1.0 * k / (j->nz - 1);
                const int64_t o = (int64_t)k + (int64_t)jj * j->nz + (int64_t)i * j->ny * j->nz;
                double e, s;
                cells_point(j->C, xf, yf, zf, &e, &s, NULL);
                j->e[o] = e;
                if (j->sabs) j->sabs[o] = s;
            }
        }
    }
    return NULL;
}

int oracle_grid_cells(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                      double rc2, int nx, int ny, int nz, double* energy, double* sum_abs,
                      int n_threads) {
    cells_t C;
    if (cells_build(&C, atoms, n_atoms, t, rep, rc2, OR_MIN_R_GRID)) return -1;
    const int nth = nthreads(n_threads, nx);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nth);
    gjob_t* jobs = (gjob_t*)calloc((size_t)nth, sizeof(gjob_t));
    for (int k = 0; k < nth; k++) {
        jobs[k].C = &C; jobs[k].nx = nx; jobs[k].ny = ny; jobs[k].nz = nz;
        jobs[k].e = energy; jobs[k].sabs = sum_abs; jobs[k].tid = k; jobs[k].nth = nth;
        pthread_create(&th[k], NULL, grid_fn, &jobs[k]);
    }
    for (int k = 0; k < nth; k++) pthread_join(th[k], NULL);
    free(th);
    free(jobs);
    cells_free(&C);
    return 0;
}

/* Widom run of oracle_henry (src/doHenry.h:70-125, src/henry.cu:157-174) with
 * the cell-list energy: same Philox points, same mask test, FP64 sums of
 * exp(-E/T) and E exp(-E/T) per contiguous chunk of insertions, chunks added
 * in order. out: sum_w, sum_ew, n_ins, max(-E/T), n_blocked. */
typedef struct {
    const cells_t* C;
    int64_t n;
    double T;
    uint64_t seed;
    const uint8_t* mask;
    int mnx, mny, mnz;
    double* energies;
    double part[5];
    int tid, nth;
} hjob_t;

static void* henry_fn(void* arg) {
    hjob_t* j = (hjob_t*)arg;
    const int64_t per = (j->n + j->nth - 1) / j->nth;
    const int64_t lo = (int64_t)j->tid * per;
    const int64_t hi = lo + per < j->n ? lo + per : j->n;
    double sw = 0.0, sew = 0.0, mx = -INFINITY, nb = 0.0;
    for (int64_t i = lo; i < hi; i++) {
        double p[3];
        oracle_insertion_point(j->seed, (uint64_t)i, p);
        if (j->mask && oracle_insertion_blocked(j->mask, j->mnx, j->mny, j->mnz, p)) {
            if (j->energies) j->energies[i] = INFINITY;
            nb += 1.0;
            continue;
        }
        double e;
        cells_point(j->C, p[0], p[1], p[2], &e, NULL, NULL);
        if (j->energies) j->energies[i] = e;
        const double w = exp(-e / j->T);
        sw += w;
        sew += e * w;
        if (-e / j->T > mx) mx = -e / j->T;
    }
    j->part[0] = sw; j->part[1] = sew; j->part[3] = mx; j->part[4] = nb;
    return NULL;
}

int oracle_henry_cells(const or_particle* atoms, int n_atoms, const double t[9],
                       const int rep[3], double rc2, double T, uint64_t seed, int64_t n_ins,
                       const uint8_t* mask, int mnx, int mny, int mnz, double* out,
                       double* energies, int n_threads) {
    cells_t C;
    if (cells_build(&C, atoms, n_atoms, t, rep, rc2, OR_MIN_R_HENRY)) return -1;
    const int nth = nthreads(n_threads, n_ins);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nth);
    hjob_t* jobs = (hjob_t*)calloc((size_t)nth, sizeof(hjob_t));
    for (int k = 0; k < nth; k++) {
        jobs[k].C = &C; jobs[k].n = n_ins; jobs[k].T = T; jobs[k].seed = seed;
        jobs[k].mask = mask; jobs[k].mnx = mnx; jobs[k].mny = mny; jobs[k].mnz = mnz;
        jobs[k].energies = energies; jobs[k].tid = k; jobs[k].nth = nth;
        pthread_create(&th[k], NULL, henry_fn, &jobs[k]);
    }
    for (int k = 0; k < nth; k++) pthread_join(th[k], NULL);
    double sw = 0.0, sew = 0.0, mx = -INFINITY, nb = 0.0;
    for (int k = 0; k < nth; k++) {
        sw += jobs[k].part[0];
        sew += jobs[k].part[1];
        if (jobs[k].part[3] > mx) mx = jobs[k].part[3];
        nb += jobs[k].part[4];
    }
    out[0] = sw; out[1] = sew; out[2] = (double)n_ins; out[3] = mx; out[4] = nb;
    free(th);
    free(jobs);
    cells_free(&C);
    return 0;
}
