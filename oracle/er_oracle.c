/*
 * er_oracle.c -- CPU restatement (FP64) of EmptyRoom's adsorption hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Nothing in the
 * product (emptyroom_b200/) links, loads or calls this file. Compiled with
 * -ffp-contract=off so every expression is evaluated in strict IEEE double,
 * in the order the reference writes it.
 */
#define _GNU_SOURCE
#include "er_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* src/computegridsheet.h:21-28 (same as src/doHenry.h:20-27). */
static inline void frac_to_cart(const double t[9], double xf, double yf, double zf,
                                double* x, double* y, double* z) {
    *x = t[0] * xf + t[1] * yf + t[2] * zf;
    *y = t[3] * xf + t[4] * yf + t[5] * zf;
    *z = t[6] * xf + t[7] * yf + t[8] * zf;
}

double oracle_point_energy(const or_particle* atoms, int n_atoms, const double t[9],
                           const int rep[3], double rc2, double min_r,
                           double xf, double yf, double zf) {
    /* src/computegridsheet.h:38-92 */
    double energy = 0.0;
    double x, y, z;
    frac_to_cart(t, xf, yf, zf, &x, &y, &z);
    const double r2min = min_r * min_r;
    for (int i = -rep[0]; i <= rep[0]; i++) {
        for (int j = -rep[1]; j <= rep[1]; j++) {
            for (int k = -rep[2]; k <= rep[2]; k++) {
                for (int a = 0; a < n_atoms; a++) {
                    double xff = atoms[a].x_f + 1.0 * i;
                    double yff = atoms[a].y_f + 1.0 * j;
                    double zff = atoms[a].z_f + 1.0 * k;
                    double xw, yw, zw;
                    frac_to_cart(t, xff, yff, zff, &xw, &yw, &zw);
                    double dx = x - xw, dy = y - yw, dz = z - zw;
                    double r2 = dx * dx + dy * dy + dz * dz;
                    r2 = (r2 > r2min) ? r2 : r2min;
                    if (r2 < rc2) {
                        double s2 = atoms[a].sig_with_adsorbate_squared / r2;
                        double s6 = s2 * s2 * s2;
                        energy += 4.0 * atoms[a].eps_with_adsorbate * s6 * (s6 - 1.0);
                    }
                }
            }
        }
    }
    return energy;
}

/* Sum of |4 eps s^6 (s^6 - 1)| over the in-cutoff terms at one point: the
 * magnitude against which FP32 rounding of the individual terms is measured. */
double oracle_point_abs_energy(const or_particle* atoms, int n_atoms, const double t[9],
                               const int rep[3], double rc2, double min_r,
                               double xf, double yf, double zf) {
    double s = 0.0;
    double x, y, z;
    frac_to_cart(t, xf, yf, zf, &x, &y, &z);
    const double r2min = min_r * min_r;
    for (int i = -rep[0]; i <= rep[0]; i++)
        for (int j = -rep[1]; j <= rep[1]; j++)
            for (int k = -rep[2]; k <= rep[2]; k++)
                for (int a = 0; a < n_atoms; a++) {
                    double xw, yw, zw;
                    frac_to_cart(t, atoms[a].x_f + 1.0 * i, atoms[a].y_f + 1.0 * j,
                                 atoms[a].z_f + 1.0 * k, &xw, &yw, &zw);
                    double dx = x - xw, dy = y - yw, dz = z - zw;
                    double r2 = dx * dx + dy * dy + dz * dz;
                    r2 = (r2 > r2min) ? r2 : r2min;
                    if (r2 < rc2) {
                        double s2 = atoms[a].sig_with_adsorbate_squared / r2;
                        double s6 = s2 * s2 * s2;
                        s += fabs(4.0 * atoms[a].eps_with_adsorbate * s6 * (s6 - 1.0));
                    }
                }
    return s;
}

/* Number of (image, atom) terms with r^2 < rc^2 at one point: the work of
 * src/computegridsheet.h:79-82 at that point. */
int64_t oracle_point_pairs(const or_particle* atoms, int n_atoms, const double t[9],
                           const int rep[3], double rc2, double min_r,
                           double xf, double yf, double zf) {
    int64_t n = 0;
    double x, y, z;
    frac_to_cart(t, xf, yf, zf, &x, &y, &z);
    const double r2min = min_r * min_r;
    for (int i = -rep[0]; i <= rep[0]; i++)
        for (int j = -rep[1]; j <= rep[1]; j++)
            for (int k = -rep[2]; k <= rep[2]; k++)
                for (int a = 0; a < n_atoms; a++) {
                    double xw, yw, zw;
                    frac_to_cart(t, atoms[a].x_f + 1.0 * i, atoms[a].y_f + 1.0 * j,
                                 atoms[a].z_f + 1.0 * k, &xw, &yw, &zw);
                    double dx = x - xw, dy = y - yw, dz = z - zw;
                    double r2 = dx * dx + dy * dy + dz * dz;
                    r2 = (r2 > r2min) ? r2 : r2min;
                    if (r2 < rc2 && atoms[a].eps_with_adsorbate != 0.0 &&
                        atoms[a].sig_with_adsorbate_squared != 0.0)
                        n++;
                }
    return n;
}

static int resolve_threads(int n_threads) {
    if (n_threads > 0) return n_threads;
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* ---- work splitting over host threads (a static interleaved partition) ---- */
typedef struct {
    const or_particle* atoms;
    int n_atoms;
    const double* t;
    const int* rep;
    double rc2, min_r;
    /* grid */
    int nx, ny, nz;
    double* out;
    uint8_t* out_mask;
    /* points */
    const double* pts;
    int64_t n_pts;
    /* henry */
    double T;
    uint64_t seed;
    const uint8_t* mask;
    int mnx, mny, mnz;
    double* energies;
    double part[5];
    int tid, nth;
} job_t;

static void* grid_worker(void* arg) {
    job_t* jb = (job_t*)arg;
    for (int i = jb->tid; i < jb->nx; i += jb->nth) {
        double xf = 1.0 * i / (jb->nx - 1);
        for (int j = 0; j < jb->ny; j++) {
            double yf = 1.0 * j / (jb->ny - 1);
            for (int k = 0; k < jb->nz; k++) {
                double zf = 1.0 * k / (jb->nz - 1);
                jb->out[(int64_t)k + (int64_t)j * jb->nz + (int64_t)i * jb->ny * jb->nz] =
                    oracle_point_energy(jb->atoms, jb->n_atoms, jb->t, jb->rep, jb->rc2,
                                        OR_MIN_R_GRID, xf, yf, zf);
            }
        }
    }
    return NULL;
}

static void run_threads(job_t* proto, int nth, void* (*fn)(void*), job_t* jobs) {
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nth);
    for (int t = 0; t < nth; t++) {
        jobs[t] = *proto;
        jobs[t].tid = t;
        jobs[t].nth = nth;
        memset(jobs[t].part, 0, sizeof(jobs[t].part));
        pthread_create(&th[t], NULL, fn, &jobs[t]);
    }
    for (int t = 0; t < nth; t++) pthread_join(th[t], NULL);
    free(th);
}

void oracle_grid(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                 double rc2, int nx, int ny, int nz, double* out, int n_threads) {
    job_t proto;
    memset(&proto, 0, sizeof(proto));
    proto.atoms = atoms; proto.n_atoms = n_atoms; proto.t = t; proto.rep = rep;
    proto.rc2 = rc2; proto.nx = nx; proto.ny = ny; proto.nz = nz; proto.out = out;
    int nth = resolve_threads(n_threads);
    if (nth > nx) nth = nx;
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * nth);
    run_threads(&proto, nth, grid_worker, jobs);
    free(jobs);
}

static void* points_worker(void* arg) {
    job_t* jb = (job_t*)arg;
    for (int64_t p = jb->tid; p < jb->n_pts; p += jb->nth) {
        if (jb->out_mask && *jb->out_mask == 2) { /* magnitude mode */
            jb->out[p] = oracle_point_abs_energy(jb->atoms, jb->n_atoms, jb->t, jb->rep, jb->rc2,
                                                 jb->min_r, jb->pts[3 * p], jb->pts[3 * p + 1],
                                                 jb->pts[3 * p + 2]);
            continue;
        }
        if (jb->out_mask) { /* count mode */
            jb->out[p] = (double)oracle_point_pairs(jb->atoms, jb->n_atoms, jb->t, jb->rep,
                                                    jb->rc2, jb->min_r, jb->pts[3 * p],
                                                    jb->pts[3 * p + 1], jb->pts[3 * p + 2]);
            continue;
        }
        jb->out[p] = oracle_point_energy(jb->atoms, jb->n_atoms, jb->t, jb->rep, jb->rc2,
                                         jb->min_r, jb->pts[3 * p], jb->pts[3 * p + 1],
                                         jb->pts[3 * p + 2]);
    }
    return NULL;
}

void oracle_points(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                   double rc2, double min_r, const double* pts, int64_t n_pts, double* out,
                   int n_threads) {
    job_t proto;
    memset(&proto, 0, sizeof(proto));
    proto.atoms = atoms; proto.n_atoms = n_atoms; proto.t = t; proto.rep = rep;
    proto.rc2 = rc2; proto.min_r = min_r; proto.pts = pts; proto.n_pts = n_pts; proto.out = out;
    int nth = resolve_threads(n_threads);
    if ((int64_t)nth > n_pts) nth = n_pts > 0 ? (int)n_pts : 1;
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * nth);
    run_threads(&proto, nth, points_worker, jobs);
    free(jobs);
}

void oracle_points_abs(const or_particle* atoms, int n_atoms, const double t[9],
                       const int rep[3], double rc2, double min_r, const double* pts,
                       int64_t n_pts, double* out, int n_threads) {
    job_t proto;
    uint8_t flag = 2;
    memset(&proto, 0, sizeof(proto));
    proto.atoms = atoms; proto.n_atoms = n_atoms; proto.t = t; proto.rep = rep;
    proto.rc2 = rc2; proto.min_r = min_r; proto.pts = pts; proto.n_pts = n_pts; proto.out = out;
    proto.out_mask = &flag;
    int nth = resolve_threads(n_threads);
    if ((int64_t)nth > n_pts) nth = n_pts > 0 ? (int)n_pts : 1;
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * nth);
    run_threads(&proto, nth, points_worker, jobs);
    free(jobs);
}

void oracle_points_pairs(const or_particle* atoms, int n_atoms, const double t[9],
                         const int rep[3], double rc2, double min_r, const double* pts,
                         int64_t n_pts, double* out, int n_threads) {
    job_t proto;
    uint8_t flag = 1;
    memset(&proto, 0, sizeof(proto));
    proto.atoms = atoms; proto.n_atoms = n_atoms; proto.t = t; proto.rep = rep;
    proto.rc2 = rc2; proto.min_r = min_r; proto.pts = pts; proto.n_pts = n_pts; proto.out = out;
    proto.out_mask = &flag;
    int nth = resolve_threads(n_threads);
    if ((int64_t)nth > n_pts) nth = n_pts > 0 ? (int)n_pts : 1;
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * nth);
    run_threads(&proto, nth, points_worker, jobs);
    free(jobs);
}

/* src/computegridsheet.h:117-164 */
static void* access_worker(void* arg) {
    job_t* jb = (job_t*)arg;
    const double* t = jb->t;
    for (int ii = jb->tid; ii < jb->nx; ii += jb->nth) {
        double xf = 1.0 * ii / (jb->nx - 1);
        for (int jj = 0; jj < jb->ny; jj++) {
            double yf = 1.0 * jj / (jb->ny - 1);
            for (int kk = 0; kk < jb->nz; kk++) {
                double zf = 1.0 * kk / (jb->nz - 1);
                double x, y, z;
                frac_to_cart(t, xf, yf, zf, &x, &y, &z);
                int overlap = 0;
                for (int i = -1; (i <= 1) && !overlap; i++)
                    for (int j = -1; (j <= 1) && !overlap; j++)
                        for (int k = -1; (k <= 1) && !overlap; k++)
                            for (int a = 0; a < jb->n_atoms; a++) {
                                double xw, yw, zw;
                                frac_to_cart(t, jb->atoms[a].x_f + i, jb->atoms[a].y_f + j,
                                             jb->atoms[a].z_f + k, &xw, &yw, &zw);
                                double dx = x - xw, dy = y - yw, dz = z - zw;
                                double r2 = dx * dx + dy * dy + dz * dz;
                                if (r2 < jb->atoms[a].sig_with_adsorbate_squared) overlap = 1;
                            }
                jb->out_mask[(int64_t)kk + (int64_t)jj * jb->nz + (int64_t)ii * jb->ny * jb->nz] =
                    overlap ? 0 : 1;
            }
        }
    }
    return NULL;
}

void oracle_accessibility(const or_particle* atoms, int n_atoms, const double t[9],
                          int nx, int ny, int nz, uint8_t* out, int n_threads) {
    job_t proto;
    memset(&proto, 0, sizeof(proto));
    proto.atoms = atoms; proto.n_atoms = n_atoms; proto.t = t;
    proto.nx = nx; proto.ny = ny; proto.nz = nz; proto.out_mask = out;
    int nth = resolve_threads(n_threads);
    if (nth > nx) nth = nx;
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * nth);
    run_threads(&proto, nth, access_worker, jobs);
    free(jobs);
}

/* ---------------- Philox4x32-10 (Salmon et al., SC'11) ---------------- */
static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* 53-bit uniform in [0,1) from two 32-bit words: (a>>5)*2^26 + (b>>6), times 2^-53. */
static inline double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

void oracle_insertion_point(uint64_t seed, uint64_t i, double out[3]) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0u, 0u};
    uint32_t r[4], s[4];
    oracle_philox4x32_10(c, key, r);
    c[2] = 1u;
    oracle_philox4x32_10(c, key, s);
    out[0] = u53(r[0], r[1]);
    out[1] = u53(r[2], r[3]);
    out[2] = u53(s[0], s[1]);
}

void oracle_insertion_points(uint64_t seed, uint64_t i0, int64_t n, double* out) {
    for (int64_t k = 0; k < n; k++) oracle_insertion_point(seed, i0 + (uint64_t)k, out + 3 * k);
}

/* An insertion is blocked when any of the 8 corners of its grid cell is set.
 * Cell lookup follows src/gcmc.cc:155-157 (floor(x_f / dx_f), dx_f = 1/(N-1)). */
int oracle_insertion_blocked(const uint8_t* mask, int nx, int ny, int nz, const double p[3]) {
    double dxf = 1.0 / (nx - 1), dyf = 1.0 / (ny - 1), dzf = 1.0 / (nz - 1);
    int i0 = (int)floor(p[0] / dxf), j0 = (int)floor(p[1] / dyf), k0 = (int)floor(p[2] / dzf);
    if (i0 > nx - 2) i0 = nx - 2;
    if (j0 > ny - 2) j0 = ny - 2;
    if (k0 > nz - 2) k0 = nz - 2;
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++)
            for (int dk = 0; dk < 2; dk++) {
                int64_t idx = (int64_t)(k0 + dk) + (int64_t)(j0 + dj) * nz +
                              (int64_t)(i0 + di) * ny * nz;
                if (mask[idx]) return 1;
            }
    return 0;
}

static void* henry_worker(void* arg) {
    job_t* jb = (job_t*)arg;
    /* contiguous chunk per thread so partial sums run in index order */
    int64_t per = (jb->n_pts + jb->nth - 1) / jb->nth;
    int64_t lo = (int64_t)jb->tid * per, hi = lo + per;
    if (hi > jb->n_pts) hi = jb->n_pts;
    double sw = 0.0, sew = 0.0, mx = -INFINITY, nb = 0.0;
    for (int64_t i = lo; i < hi; i++) {
        double p[3];
        oracle_insertion_point(jb->seed, (uint64_t)i, p);
        if (jb->mask && oracle_insertion_blocked(jb->mask, jb->mnx, jb->mny, jb->mnz, p)) {
            if (jb->energies) jb->energies[i] = INFINITY;
            nb += 1.0;
            continue;
        }
        double e = oracle_point_energy(jb->atoms, jb->n_atoms, jb->t, jb->rep, jb->rc2,
                                       OR_MIN_R_HENRY, p[0], p[1], p[2]);
        if (jb->energies) jb->energies[i] = e;
        double w = exp(-e / jb->T); /* src/doHenry.h:107 */
        sw += w;
        sew += e * w;
        if (-e / jb->T > mx) mx = -e / jb->T;
    }
    jb->part[0] = sw; jb->part[1] = sew; jb->part[3] = mx; jb->part[4] = nb;
    return NULL;
}

void oracle_henry(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                  double rc2, double T, uint64_t seed, int64_t n_ins,
                  const uint8_t* mask, int mnx, int mny, int mnz,
                  double* out, double* energies, int n_threads) {
    job_t proto;
    memset(&proto, 0, sizeof(proto));
    proto.atoms = atoms; proto.n_atoms = n_atoms; proto.t = t; proto.rep = rep;
    proto.rc2 = rc2; proto.T = T; proto.seed = seed; proto.n_pts = n_ins;
    proto.mask = mask; proto.mnx = mnx; proto.mny = mny; proto.mnz = mnz;
    proto.energies = energies;
    int nth = resolve_threads(n_threads);
    if ((int64_t)nth > n_ins) nth = n_ins > 0 ? (int)n_ins : 1;
    job_t* jobs = (job_t*)malloc(sizeof(job_t) * nth);
    run_threads(&proto, nth, henry_worker, jobs);
    double sw = 0.0, sew = 0.0, mx = -INFINITY, nb = 0.0;
    for (int t2 = 0; t2 < nth; t2++) {
        sw += jobs[t2].part[0];
        sew += jobs[t2].part[1];
        if (jobs[t2].part[3] > mx) mx = jobs[t2].part[3];
        nb += jobs[t2].part[4];
    }
    free(jobs);
    out[0] = sw; out[1] = sew; out[2] = (double)n_ins; out[3] = mx; out[4] = nb;
}

/* ---------------- pocket blocking: src/pocketblocking.cc:126-391 ---------------- */
typedef struct { int from, to, dir; } conn_t;
typedef struct { int i, j, k; } uc_t;

static int64_t gidx(int i, int j, int k, int ny, int nz) {
    return (int64_t)k + (int64_t)j * nz + (int64_t)i * ny * nz; /* pocketblocking.cc:10-13 */
}

/* pocketblocking.cc:103-124 */
static void note_connection(conn_t** c, int* n, int* cap, int from, int to, int dir) {
    for (int q = 0; q < *n; q++) {
        if ((*c)[q].to == to && (*c)[q].from == from) {
            if (to == from || dir == (*c)[q].dir) return;
        }
    }
    if (*n == *cap) {
        *cap = *cap ? 2 * *cap : 64;
        *c = (conn_t*)realloc(*c, sizeof(conn_t) * (*cap));
    }
    (*c)[*n].from = from; (*c)[*n].to = to; (*c)[*n].dir = dir;
    (*n)++;
}

/* Iterative form of recursively_navigate_connections (pocketblocking.cc:39-100):
 * the same visit of every edge reachable from `start`, with the same
 * self-loop and unit-cell consistency tests. */
static int segment_is_channel(int start, int n_seg, const conn_t* c, int nc,
                              char* seg_vis, char* edge_vis, uc_t* uc, int* stack, int* pos) {
    memset(seg_vis, 0, n_seg);
    memset(edge_vis, 0, nc);
    for (int s = 0; s < n_seg; s++) { uc[s].i = uc[s].j = uc[s].k = 0; }
    int found = 0, top = 0;
    stack[top] = start; pos[top] = 0; top++;
    seg_vis[start] = 1;
    while (top > 0) {
        int seg = stack[top - 1];
        int q = pos[top - 1];
        if (q >= nc) { top--; continue; }
        pos[top - 1] = q + 1;
        if (edge_vis[q]) continue;
        if (c[q].to == seg && c[q].from == seg) {
            edge_vis[q] = 1;
            found = 1;
        } else if (c[q].to == seg || c[q].from == seg) {
            edge_vis[q] = 1;
            int other = c[q].to, dir = c[q].dir;
            if (c[q].to == seg) { other = c[q].from; dir = -dir; }
            uc_t nu = uc[seg];
            if (dir == 1) nu.i++;
            if (dir == 2) nu.j++;
            if (dir == 3) nu.k++;
            if (dir == -1) nu.i--;
            if (dir == -2) nu.j--;
            if (dir == -3) nu.k--;
            if (!seg_vis[other]) {
                uc[other] = nu;
                seg_vis[other] = 1;
                stack[top] = other; pos[top] = 0; top++;
            } else {
                uc_t ou = uc[other];
                if (nu.i != ou.i || nu.j != ou.j || nu.k != ou.k) found = 1;
            }
        }
    }
    return found;
}

int oracle_block_pockets(double* grid, int nx, int ny, int nz, double temperature,
                         int* segment_out) {
    int64_t n = (int64_t)nx * ny * nz;
    double thr = 15.0 * temperature; /* pocketblocking.cc:130 */
    int* seg = (int*)malloc(sizeof(int) * n);
    char* found = (char*)malloc(n);
    for (int64_t p = 0; p < n; p++) {
        if (grid[p] >= thr) { found[p] = 1; seg[p] = -1; }
        else found[p] = 0;
    }
    /* flood fill, pocketblocking.cc:152-251 */
    int n_seg = 0;
    int64_t cap = 1024, top = 0;
    int64_t* st = (int64_t*)malloc(sizeof(int64_t) * cap);
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                int64_t g = gidx(i, j, k, ny, nz);
                if (found[g]) continue;
                n_seg++;
                top = 0;
                st[top++] = g;
                while (top > 0) {
                    int64_t q = st[--top];
                    found[q] = 1;
                    seg[q] = n_seg - 1;
                    int qk = (int)(q % nz), qj = (int)((q / nz) % ny), qi = (int)(q / ((int64_t)ny * nz));
                    int64_t nb[6];
                    int m = 0;
                    if (qi != 0) nb[m++] = gidx(qi - 1, qj, qk, ny, nz);
                    if (qi != nx - 1) nb[m++] = gidx(qi + 1, qj, qk, ny, nz);
                    if (qj != 0) nb[m++] = gidx(qi, qj - 1, qk, ny, nz);
                    if (qj != ny - 1) nb[m++] = gidx(qi, qj + 1, qk, ny, nz);
                    if (qk != 0) nb[m++] = gidx(qi, qj, qk - 1, ny, nz);
                    if (qk != nz - 1) nb[m++] = gidx(qi, qj, qk + 1, ny, nz);
                    for (int u = 0; u < m; u++) {
                        if (!found[nb[u]]) {
                            if (top == cap) { cap *= 2; st = (int64_t*)realloc(st, sizeof(int64_t) * cap); }
                            st[top++] = nb[u];
                        }
                    }
                }
            }
    free(st);
    free(found);
    /* periodic face graph, pocketblocking.cc:277-321 */
    conn_t* c = NULL;
    int nc = 0, ccap = 0;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            int a = seg[gidx(0, j, k, ny, nz)], b = seg[gidx(nx - 1, j, k, ny, nz)];
            if (a != -1 && b != -1) note_connection(&c, &nc, &ccap, b, a, 1);
        }
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            int a = seg[gidx(i, 0, k, ny, nz)], b = seg[gidx(i, ny - 1, k, ny, nz)];
            if (a != -1 && b != -1) note_connection(&c, &nc, &ccap, b, a, 2);
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            int a = seg[gidx(i, j, 0, ny, nz)], b = seg[gidx(i, j, nz - 1, ny, nz)];
            if (a != -1 && b != -1) note_connection(&c, &nc, &ccap, b, a, 3);
        }
    /* classification, pocketblocking.cc:330-365 */
    char* is_pocket = (char*)calloc(n_seg > 0 ? n_seg : 1, 1);
    char* seg_vis = (char*)malloc(n_seg > 0 ? n_seg : 1);
    char* edge_vis = (char*)malloc(nc > 0 ? nc : 1);
    uc_t* uc = (uc_t*)malloc(sizeof(uc_t) * (n_seg > 0 ? n_seg : 1));
    int* stack = (int*)malloc(sizeof(int) * (n_seg + 1));
    int* pos = (int*)malloc(sizeof(int) * (n_seg + 1));
    int n_pockets = 0;
    for (int s = 0; s < n_seg; s++) {
        if (!segment_is_channel(s, n_seg, c, nc, seg_vis, edge_vis, uc, stack, pos)) {
            is_pocket[s] = 1;
            n_pockets++;
        }
    }
    /* overwrite, pocketblocking.cc:373-382 */
    for (int64_t p = 0; p < n; p++)
        if (seg[p] >= 0 && is_pocket[seg[p]]) grid[p] = 1e13;
    if (segment_out) memcpy(segment_out, seg, sizeof(int) * n);
    free(is_pocket); free(seg_vis); free(edge_vis); free(uc); free(stack); free(pos);
    free(c);
    free(seg);
    return n_pockets;
}

/* ------------------------------------------------------------------------
 * GCMC trilinear lookup, src/gcmc.cc:74-77 and :137-177 (see er_oracle.h). */
static double gi_wrap1(double x) { return x - 1.0 * floor(x / 1.0); }

void oracle_grid_interp(const double* grid, int nx, int ny, int nz, const double* pts,
                        int64_t n, double* out) {
    const double dx = 1.0 / (nx - 1), dy = 1.0 / (ny - 1), dz = 1.0 / (nz - 1);
    for (int64_t q = 0; q < n; ++q) {
        const double x = gi_wrap1(pts[3 * q]), y = gi_wrap1(pts[3 * q + 1]),
                     z = gi_wrap1(pts[3 * q + 2]);
        int i = (int)floor(x / dx), j = (int)floor(y / dy), k = (int)floor(z / dz);
        if (i > nx - 2) i = nx - 2;
        if (j > ny - 2) j = ny - 2;
        if (k > nz - 2) k = nz - 2;
        const double xd = (x - i * dx) / dx;
        const double yd = (y - j * dy) / dy;
        const double zd = (z - k * dz) / dz;
#define G(a, b, c) grid[(size_t)(c) + (size_t)(b) * nz + (size_t)(a) * ny * nz]
        const double c00 = G(i, j, k) * (1.0 - xd) + xd * G(i + 1, j, k);
        const double c10 = G(i, j + 1, k) * (1.0 - xd) + xd * G(i + 1, j + 1, k);
        const double c01 = G(i, j, k + 1) * (1.0 - xd) + xd * G(i + 1, j, k + 1);
        const double c11 = G(i, j + 1, k + 1) * (1.0 - xd) + xd * G(i + 1, j + 1, k + 1);
#undef G
        const double c0 = c00 * (1.0 - yd) + c10 * yd;
        const double c1 = c01 * (1.0 - yd) + c11 * yd;
        out[q] = c0 * (1.0 - zd) + c1 * zd;
    }
}
