/*
 * er_oracle_synth.c -- the seeded synthetic frameworks of the benchmark
 * workloads, generated without the library under test.
 *
 * TEST INFRASTRUCTURE ONLY (see er_oracle.h). The benchmark's reference arm
 * times the reference's CPU code on the same frameworks as the GPU arm, and
 * must not load the library it is compared with; these functions restate the
 * library's host generators (cell matrices, replication factors, random
 * sequential addition of atoms) so that the reference arm builds the same
 * inputs bit for bit. tests/test_oracle_pin.py checks that they agree with
 * the library's er_cell_matrices, er_replication_factors and
 * er_synth_positions.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "er_oracle.h"

/* Cell matrix, inverse and volume from lengths and angles (degrees): the
 * formulas and expression order of src/Framework.cc:35-37, 113-142. */
int oracle_cell_matrices(double a, double b, double c, double alpha_deg, double beta_deg,
                         double gamma_deg, double t[9], double inv[9], double* volume) {
    const double al = alpha_deg * M_PI / 180.0;
    const double be = beta_deg * M_PI / 180.0;
    const double ga = gamma_deg * M_PI / 180.0;
    const double arg = 1.0 - pow(cos(al), 2.0) - pow(cos(be), 2) - pow(cos(ga), 2) +
                       2 * cos(al) * cos(be) * cos(ga);
    if (!(a > 0) || !(b > 0) || !(c > 0) || !(arg > 0) || sin(ga) == 0.0) return -1;
    const double v = sqrt(arg);
    if (volume) *volume = v * a * b * c;
    if (t) {
        t[0] = a; t[1] = b * cos(ga); t[2] = c * cos(be);
        t[3] = 0.0; t[4] = b * sin(ga); t[5] = c * (cos(al) - cos(be) * cos(ga)) / sin(ga);
        t[6] = 0.0; t[7] = 0.0; t[8] = c * v / sin(ga);
    }
    if (inv) {
        inv[0] = 1.0 / a;
        inv[1] = -cos(ga) / a / sin(ga);
        inv[2] = (cos(al) * cos(ga) - cos(be)) / (a * v * sin(ga));
        inv[3] = 0.0;
        inv[4] = 1.0 / b / sin(ga);
        inv[5] = (cos(be) * cos(ga) - cos(al)) / (b * v * sin(ga));
        inv[6] = 0.0;
        inv[7] = 0.0;
        inv[8] = sin(ga) / (c * v);
    }
    return 0;
}

static void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* Perpendicular widths of the cell: volume over the area of each face. */
static void widths(const double t[9], double w[3]) {
    const double a[3] = {t[0], t[3], t[6]}, b[3] = {t[1], t[4], t[7]}, c[3] = {t[2], t[5], t[8]};
    double bc[3], ca[3], ab[3];
    cross3(b, c, bc);
    cross3(c, a, ca);
    cross3(a, b, ab);
    const double vol = fabs(a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2]);
    w[0] = vol / sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    w[1] = vol / sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]);
    w[2] = vol / sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2]);
}

/* floor(factor * rc / w_i) + 1 images per side: every image within rc of the
 * unit cell is summed (the .uc files of src/readsettings.h:243-274). */
int oracle_replication_factors(const double t[9], double r_cutoff, int factor, int rep[3]) {
    if (!(r_cutoff > 0) || factor < 1) return -1;
    double w[3];
    widths(t, w);
    for (int k = 0; k < 3; k++) {
        if (!(w[k] > 0)) return -1;
        rep[k] = (int)floor(factor * r_cutoff / w[k]) + 1;
    }
    return 0;
}

static inline double u53s(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* Random sequential addition: attempt k draws a fractional position from the
 * Philox4x32-10 stream of `seed` (counters (k, lane 7) and (k, lane 8)) and
 * keeps it when no kept atom is within d_min under the 27 nearest periodic
 * images (bins of at least d_min per axis). Returns 0, or -1 when n_atoms
 * could not be placed within the attempt budget. */
int oracle_synth_positions(uint64_t seed, const double t[9], int n_atoms, double d_min,
                           double* frac) {
    if (n_atoms < 0 || d_min < 0) return -1;
    double w[3];
    widths(t, w);
    const double dm2 = d_min * d_min;
    int nb[3];
    for (int k = 0; k < 3; k++) {
        nb[k] = d_min > 0 ? (int)floor(w[k] / (d_min > 1e-3 ? d_min : 1e-3)) : 1;
        if (nb[k] < 1) nb[k] = 1;
        if (nb[k] > 256) nb[k] = 256;
    }
    const size_t nbin = (size_t)nb[0] * nb[1] * nb[2];
    int* head = (int*)malloc(sizeof(int) * nbin);
    int* next = (int*)malloc(sizeof(int) * (size_t)(n_atoms > 0 ? n_atoms : 1));
    for (size_t q = 0; q < nbin; q++) head[q] = -1;
    const int64_t max_attempts = (int64_t)n_atoms * 2000 + 100000;
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    int n = 0;
    for (int64_t att = 0; n < n_atoms && att < max_attempts; att++) {
        uint32_t c1[4] = {(uint32_t)att, (uint32_t)((uint64_t)att >> 32), 7u, 0u};
        uint32_t c2[4] = {(uint32_t)att, (uint32_t)((uint64_t)att >> 32), 8u, 0u};
        uint32_t r[4], r2[4];
        oracle_philox4x32_10(c1, key, r);
        oracle_philox4x32_10(c2, key, r2);
        const double f[3] = {u53s(r[0], r[1]), u53s(r[2], r[3]), u53s(r2[0], r2[1])};
        int b[3];
        for (int k = 0; k < 3; k++) {
            b[k] = (int)(f[k] * nb[k]);
            if (b[k] > nb[k] - 1) b[k] = nb[k] - 1;
        }
        int ok = 1;
        if (d_min > 0) {
            for (int di = -1; di <= 1 && ok; di++)
                for (int dj = -1; dj <= 1 && ok; dj++)
                    for (int dk = -1; dk <= 1 && ok; dk++) {
                        const int bi = (b[0] + di + nb[0]) % nb[0];
                        const int bj = (b[1] + dj + nb[1]) % nb[1];
                        const int bk = (b[2] + dk + nb[2]) % nb[2];
                        for (int q = head[((size_t)bi * nb[1] + bj) * nb[2] + bk]; q >= 0 && ok;
                             q = next[q]) {
                            double d0 = f[0] - frac[3 * q], d1 = f[1] - frac[3 * q + 1],
                                   d2 = f[2] - frac[3 * q + 2];
                            d0 -= floor(d0 + 0.5);
                            d1 -= floor(d1 + 0.5);
                            d2 -= floor(d2 + 0.5);
                            for (int ii = -1; ii <= 1 && ok; ii++)
                                for (int jj = -1; jj <= 1 && ok; jj++)
                                    for (int kk = -1; kk <= 1 && ok; kk++) {
                                        const double e0 = d0 + ii, e1 = d1 + jj, e2 = d2 + kk;
                                        const double x = t[0] * e0 + t[1] * e1 + t[2] * e2;
                                        const double y = t[3] * e0 + t[4] * e1 + t[5] * e2;
                                        const double z = t[6] * e0 + t[7] * e1 + t[8] * e2;
                                        if (x * x + y * y + z * z < dm2) ok = 0;
                                    }
                        }
                    }
        }
        if (!ok) continue;
        frac[3 * n] = f[0];
        frac[3 * n + 1] = f[1];
        frac[3 * n + 2] = f[2];
        const size_t bin = ((size_t)b[0] * nb[1] + b[1]) * nb[2] + b[2];
        next[n] = head[bin];
        head[bin] = n;
        n++;
    }
    free(head);
    free(next);
    return n == n_atoms ? 0 : -1;
}
