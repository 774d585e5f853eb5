/*
 * ref_shim.cc -- runs the reference's own code on the host, as the parity
 * checker for the oracle restatement and, when built, as the CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles this file against the
 * reference's unmodified sources where they lie (src/computegridsheet.h,
 * src/pocketblocking.cc, src/Framework.cc, src/Forcefield.cc) into
 * oracle/_ref/libref.so. No reference source is copied into this repository:
 * the headers are included from the reference tree at build time.
 *
 * The CUDA kernels of src/computegridsheet.h are compiled as plain host
 * functions: __global__/__device__ expand to nothing and threadIdx/blockIdx/
 * blockDim are thread-local host variables set by the driver loops below,
 * which walk the reference's own 16x16 block decomposition
 * (src/writegrid.cu:205-206) for every x-sheet (src/writegrid.cu:219-226).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <string>
#include <vector>

#define __global__
#define __device__
struct ShimDim3 {
    unsigned x, y, z;
};
static thread_local ShimDim3 threadIdx, blockIdx, blockDim;

#include "datatypes.h"
#include "computegridsheet.h"
#include "Framework.h"
#include "Forcefield.h"
#include "pocketblocking.h"

namespace {

struct SheetJob {
    const FrameworkParticle* atoms;
    GridParameters* params;
    std::vector<double>* yaxis;
    std::vector<double>* zaxis;
    std::vector<double>* xaxis;
    double* out;  // n_sheets*ny*nz
    int accessibility;
    const int* sheets;  // x indices to compute (NULL: all, out index = x index)
    int n_sheets;
    int tid, nth;
};

void* sheet_worker(void* arg) {
    SheetJob* jb = static_cast<SheetJob*>(arg);
    GridParameters& p = *jb->params;
    const int S = 16;  // SQRT_N_THREADS, src/writegrid.cu:18
    blockDim.x = S; blockDim.y = S; blockDim.z = 1;
    std::vector<double> sheet((size_t)p.N_y * p.N_z);
    for (int s_ = jb->tid; s_ < jb->n_sheets; s_ += jb->nth) {
        const int i = jb->sheets ? jb->sheets[s_] : s_;
        double xf = (*jb->xaxis)[i];
        for (int by = 0; by < p.N_y / S + 1; by++)
            for (int bz = 0; bz < p.N_z / S + 1; bz++)
                for (int ty = 0; ty < S; ty++)
                    for (int tz = 0; tz < S; tz++) {
                        blockIdx.x = bz; blockIdx.y = by;
                        threadIdx.x = tz; threadIdx.y = ty;
                        if (jb->accessibility)
                            ComputeGridSheetAccessibleOrNot(jb->zaxis->data(), jb->yaxis->data(),
                                                            sheet.data(),
                                                            const_cast<FrameworkParticle*>(jb->atoms),
                                                            p, xf);
                        else
                            ComputeGridSheet(jb->zaxis->data(), jb->yaxis->data(), sheet.data(),
                                             const_cast<FrameworkParticle*>(jb->atoms), p, xf);
                    }
        memcpy(jb->out + (size_t)s_ * p.N_y * p.N_z, sheet.data(),
               sizeof(double) * (size_t)p.N_y * p.N_z);
    }
    return nullptr;
}

void run_grid(const double* particles, int n_atoms, const double* t, const int* rep, double rc2,
              int nx, int ny, int nz, double* out, int n_threads, int accessibility,
              const int* sheets = nullptr, int n_sheets = -1) {
    if (n_sheets < 0) n_sheets = nx;
    GridParameters p;
    p.N_framework_atoms = n_atoms;
    p.N_x = nx; p.N_y = ny; p.N_z = nz;
    p.replication_factor_a = rep[0];
    p.replication_factor_b = rep[1];
    p.replication_factor_c = rep[2];
    p.r_cutoff_squared = rc2;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) p.t_matrix[a][b] = t[3 * a + b];
    std::vector<FrameworkParticle> atoms(n_atoms);
    for (int a = 0; a < n_atoms; a++) {
        atoms[a].x_f = particles[5 * a + 0];
        atoms[a].y_f = particles[5 * a + 1];
        atoms[a].z_f = particles[5 * a + 2];
        atoms[a].eps_with_adsorbate = particles[5 * a + 3];
        atoms[a].sig_with_adsorbate_squared = particles[5 * a + 4];
    }
    // grid axes, src/writegrid.cu:122-127
    std::vector<double> xa(nx), ya(ny), za(nz);
    for (int i = 0; i < nx; i++) xa[i] = 1.0 * i / (nx - 1);
    for (int i = 0; i < ny; i++) ya[i] = 1.0 * i / (ny - 1);
    for (int i = 0; i < nz; i++) za[i] = 1.0 * i / (nz - 1);
    int nth = n_threads > 0 ? n_threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nth > n_sheets) nth = n_sheets;
    if (nth < 1) nth = 1;
    std::vector<SheetJob> jobs(nth);
    std::vector<pthread_t> th(nth);
    for (int k = 0; k < nth; k++) {
        jobs[k] = SheetJob{atoms.data(), &p, &ya, &za, &xa, out, accessibility, sheets, n_sheets,
                           k, nth};
        pthread_create(&th[k], nullptr, sheet_worker, &jobs[k]);
    }
    for (int k = 0; k < nth; k++) pthread_join(th[k], nullptr);
}

struct PointJob {
    const FrameworkParticle* atoms;
    const GridParameters* params;
    const double* pts;
    int64_t n_pts;
    double* out;
    int tid, nth;
};

// ComputeGridSheet on one-point axes: thread (0, 0) of block (0, 0) computes
// the point (pts[3i], pts[3i+1], pts[3i+2]) -- the reference's LJ routine at
// an arbitrary point, e.g. a Widom insertion (src/doHenry.h:70-98 is the same
// sum with min_r 1e-16 instead of 1e-12).
void* point_worker(void* arg) {
    PointJob* jb = static_cast<PointJob*>(arg);
    GridParameters p = *jb->params;
    p.N_x = 1; p.N_y = 1; p.N_z = 1;
    blockDim.x = 16; blockDim.y = 16; blockDim.z = 1;
    blockIdx.x = blockIdx.y = blockIdx.z = 0;
    threadIdx.x = threadIdx.y = threadIdx.z = 0;
    for (int64_t i = jb->tid; i < jb->n_pts; i += jb->nth) {
        double y = jb->pts[3 * i + 1], z = jb->pts[3 * i + 2], e = 0.0;
        ComputeGridSheet(&z, &y, &e, const_cast<FrameworkParticle*>(jb->atoms), p,
                         jb->pts[3 * i]);
        jb->out[i] = e;
    }
    return nullptr;
}

}  // namespace

extern "C" {

/* The reference's ComputeGridSheet evaluated at n_pts fractional points
 * (n_pts x 3), threads over points; out[i] = energy at point i. */
void ref_points(const double* particles, int n_atoms, const double* t, const int* rep,
                double rc2, const double* pts, int64_t n_pts, double* out, int n_threads) {
    GridParameters p;
    p.N_framework_atoms = n_atoms;
    p.N_x = p.N_y = p.N_z = 1;
    p.replication_factor_a = rep[0];
    p.replication_factor_b = rep[1];
    p.replication_factor_c = rep[2];
    p.r_cutoff_squared = rc2;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) p.t_matrix[a][b] = t[3 * a + b];
    std::vector<FrameworkParticle> atoms(n_atoms);
    for (int a = 0; a < n_atoms; a++) {
        atoms[a].x_f = particles[5 * a + 0];
        atoms[a].y_f = particles[5 * a + 1];
        atoms[a].z_f = particles[5 * a + 2];
        atoms[a].eps_with_adsorbate = particles[5 * a + 3];
        atoms[a].sig_with_adsorbate_squared = particles[5 * a + 4];
    }
    int nth = n_threads > 0 ? n_threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if ((int64_t)nth > n_pts) nth = (int)(n_pts > 0 ? n_pts : 1);
    std::vector<PointJob> jobs(nth);
    std::vector<pthread_t> th(nth);
    for (int k = 0; k < nth; k++) {
        jobs[k] = PointJob{atoms.data(), &p, pts, n_pts, out, k, nth};
        pthread_create(&th[k], nullptr, point_worker, &jobs[k]);
    }
    for (int k = 0; k < nth; k++) pthread_join(th[k], nullptr);
}

/* particles: n x 5 doubles in FrameworkParticle order (x_f, y_f, z_f, eps, sig2);
 * t: row-major 3x3; rep: replication factors; out: nx*ny*nz doubles. */
void ref_grid(const double* particles, int n_atoms, const double* t, const int* rep, double rc2,
              int nx, int ny, int nz, double* out, int n_threads) {
    run_grid(particles, n_atoms, t, rep, rc2, nx, ny, nz, out, n_threads, 0);
}

/* ComputeGridSheet for the listed x-sheets only; out holds n_sheets*ny*nz doubles. */
void ref_grid_sheets(const double* particles, int n_atoms, const double* t, const int* rep,
                     double rc2, int nx, int ny, int nz, const int* sheets, int n_sheets,
                     double* out, int n_threads) {
    run_grid(particles, n_atoms, t, rep, rc2, nx, ny, nz, out, n_threads, 0, sheets, n_sheets);
}

/* ComputeGridSheetAccessibleOrNot over the whole grid; out holds 0.0 / 1.0. */
void ref_accessibility(const double* particles, int n_atoms, const double* t, int nx, int ny,
                       int nz, double* out, int n_threads) {
    int rep[3] = {1, 1, 1};
    run_grid(particles, n_atoms, t, rep, 0.0, nx, ny, nz, out, n_threads, 1);
}

/* FindAndBlockPockets (src/pocketblocking.cc:126) on a caller-owned grid. */
int ref_block_pockets(double* grid, int nx, int ny, int nz, double temperature) {
    GridInfo gi;
    gi.N_x = nx; gi.N_y = ny; gi.N_z = nz;
    gi.numtotalpts = nx * ny * nz;
    gi.dx_f = 1.0 / (nx - 1); gi.dy_f = 1.0 / (ny - 1); gi.dz_f = 1.0 / (nz - 1);
    GCMCParameters p;
    p.verbose = false;
    p.debugmode = false;
    return FindAndBlockPockets(grid, gi, temperature, p);
}

/* Framework (src/Framework.cc:13) constructed from <root>/data/structures/<name>.cssr
 * and <root>/data/masses.def. out: a,b,c, alpha,beta,gamma (radians), volume,
 * density, t_matrix[9], inv_t_matrix[9] (24 doubles). frac: noatoms x 3.
 * Returns noatoms. Changes the working directory to root for the call. */
int ref_load_framework(const char* root, const char* name, double* out, double* frac,
                       int max_atoms) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return -1;
    if (chdir(root) != 0) return -1;
    Framework f(name);
    if (chdir(cwd) != 0) return -1;
    out[0] = f.a; out[1] = f.b; out[2] = f.c;
    out[3] = f.alpha; out[4] = f.beta; out[5] = f.gamma;
    out[6] = f.volume_unitcell; out[7] = f.density;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            out[8 + 3 * a + b] = f.t_matrix[a][b];
            out[17 + 3 * a + b] = f.inv_t_matrix[a][b];
        }
    for (int a = 0; a < f.noatoms && a < max_atoms; a++) {
        frac[3 * a] = f.x_f[a];
        frac[3 * a + 1] = f.y_f[a];
        frac[3 * a + 2] = f.z_f[a];
    }
    return f.noatoms;
}

/* Forcefield (src/Forcefield.cc:15) from <root>/data/forcefields/<name>.def.
 * eps/sig receive up to max entries. Returns numinteractions. */
int ref_load_forcefield(const char* root, const char* name, double* eps, double* sig, int max) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return -1;
    if (chdir(root) != 0) return -1;
    Forcefield f(name);
    if (chdir(cwd) != 0) return -1;
    for (int k = 0; k < f.numinteractions && k < max; k++) {
        eps[k] = f.epsilon[k];
        sig[k] = f.sigma[k];
    }
    return f.numinteractions;
}

}  // extern "C"
