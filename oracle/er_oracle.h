/*
 * er_oracle.h -- CPU restatement (FP64) of EmptyRoom's adsorption hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path
 * (tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg call it);
 * it is never linked into, called by, or measured as the product.
 *
 * Each function names the reference file:line it restates (paths are
 * relative to the CorySimon/EmptyRoom project root). Parity of this
 * restatement against the reference's own code, compiled from its sources
 * by oracle/Makefile into oracle/_ref/, is pinned by tests/test_oracle_pin.py
 * and by the golden vectors in tests/golden/.
 */
#ifndef ER_ORACLE_H_
#define ER_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order and types as FrameworkParticle (src/datatypes.h:20-28). */
typedef struct {
    double x_f, y_f, z_f;
    double eps_with_adsorbate;
    double sig_with_adsorbate_squared;
} or_particle;

/* Clamp constants: src/computegridsheet.h:19 (grid) and src/doHenry.h:15 (Widom). */
#define OR_MIN_R_GRID 1e-12
#define OR_MIN_R_HENRY 1e-16

/* Energy (K) at one fractional point: the image x atom loop of
 * src/computegridsheet.h:54-92 (identical to src/doHenry.h:70-98 apart from
 * the clamp radius). Strict IEEE, evaluation order as written there. */
double oracle_point_energy(const or_particle* atoms, int n_atoms, const double t[9],
                           const int rep[3], double rc2, double min_r,
                           double xf, double yf, double zf);

/* Whole grid with axes i/(N-1) (src/writegrid.cu:122-127), layout
 * out[k + j*nz + i*ny*nz] (src/writegrid.cu:260-269 written sheet by sheet).
 * Sheets are split over n_threads host threads (0 = all cores). */
void oracle_grid(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                 double rc2, int nx, int ny, int nz, double* out, int n_threads);

/* Energies at an explicit list of fractional points (n x 3), n_threads as above. */
void oracle_points(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                   double rc2, double min_r, const double* pts, int64_t n_pts, double* out,
                   int n_threads);

/* Number of in-cutoff (r^2 < rc^2) terms with nonzero epsilon and sigma at each
 * point: the algorithmic work count of the pair sum. */
int64_t oracle_point_pairs(const or_particle* atoms, int n_atoms, const double t[9],
                           const int rep[3], double rc2, double min_r,
                           double xf, double yf, double zf);
void oracle_points_pairs(const or_particle* atoms, int n_atoms, const double t[9],
                         const int rep[3], double rc2, double min_r, const double* pts,
                         int64_t n_pts, double* out, int n_threads);

/* Sum over in-cutoff terms of |4 eps s^6 (s^6 - 1)| at each point: the scale of
 * the FP32 rounding error of the pair sum. */
double oracle_point_abs_energy(const or_particle* atoms, int n_atoms, const double t[9],
                               const int rep[3], double rc2, double min_r,
                               double xf, double yf, double zf);
void oracle_points_abs(const or_particle* atoms, int n_atoms, const double t[9],
                       const int rep[3], double rc2, double min_r, const double* pts,
                       int64_t n_pts, double* out, int n_threads);

/* Hard-sphere accessibility (1 accessible, 0 overlap) with images fixed to
 * +-1 and no cutoff: src/computegridsheet.h:101-165. */
void oracle_accessibility(const or_particle* atoms, int n_atoms, const double t[9],
                          int nx, int ny, int nz, uint8_t* out, int n_threads);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): 10 rounds, multipliers 0xD2511F53/0xCD9E8D57,
 * Weyl key increments 0x9E3779B9/0xBB67AE85. */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Fractional insertion point i of stream `seed`, each coordinate uniform in
 * [0,1) with 53 random bits. Replaces the MTGP32 darts of src/doHenry.h:53-55. */
void oracle_insertion_point(uint64_t seed, uint64_t i, double out[3]);
/* Points i0 .. i0 + n - 1 of stream seed into out (n x 3). */
void oracle_insertion_points(uint64_t seed, uint64_t i0, int64_t n, double* out);

/* Widom statistics over insertions [0, n_ins) of stream `seed`
 * (src/doHenry.h:53-125 per insertion, src/henry.cu:157-174 reduction).
 * mask (may be NULL) is a pocket-block mask on an mnx x mny x mnz grid with
 * axes i/(N-1): an insertion is blocked when any of the 8 surrounding
 * corners is set, and then contributes w = 0.
 * out[0] = sum w, out[1] = sum E w, out[2] = n_ins, out[3] = max(-E/T),
 * out[4] = number of blocked insertions. energies (may be NULL) receives E. */
void oracle_henry(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                  double rc2, double T, uint64_t seed, int64_t n_ins,
                  const uint8_t* mask, int mnx, int mny, int mnz,
                  double* out, double* energies, int n_threads);

/* Pocket blocking, src/pocketblocking.cc:126-391: threshold E >= 15 T,
 * non-periodic 6-connected flood fill in scan order, periodic face graph,
 * DFS channel/pocket classification, pocket points overwritten with 1e13.
 * segment_out (may be NULL) receives the segment id per point (-1 blocked).
 * Returns the number of pockets. */
int oracle_block_pockets(double* grid, int nx, int ny, int nz, double temperature,
                         int* segment_out);

/* GCMC guest-framework energy by trilinear interpolation of a grid,
 * src/gcmc.cc:145-177, at WrapToInterval(x, 1) of each coordinate
 * (src/gcmc.cc:74-77, applied at the call sites :191-194); grid spacing
 * 1 / (N - 1) (src/gcmc.cc:343), layout k + j nz + i ny nz. The lower corner
 * index is clamped to N - 2 (the reference reads past the grid when x / dx
 * rounds up to N - 1 for x just below 1). */
void oracle_grid_interp(const double* grid, int nx, int ny, int nz, const double* pts,
                        int64_t n, double* out);

/* An insertion is blocked when any of the 8 corners of its mask cell is set
 * (cell lookup of src/gcmc.cc:155-157). */
int oracle_insertion_blocked(const uint8_t* mask, int nx, int ny, int nz, const double p[3]);

/* ---- er_oracle_cells.c: the same FP64 sums over a Cartesian cell list ----
 * Every term and the set of terms equal the image loop's; only the order of
 * the additions differs. Return 0, or -1 when memory ran out. */
/* Per point (n x 3 fractional): energy, sum |term| and in-cutoff term count
 * (each output may be NULL). */
int oracle_points_cells(const or_particle* atoms, int n_atoms, const double t[9],
                        const int rep[3], double rc2, double min_r, const double* pts,
                        int64_t n_pts, double* energy, double* sum_abs, double* n_terms,
                        int n_threads);
/* Whole grid (axes i/(N-1), layout k + j nz + i ny nz); sum_abs may be NULL. */
int oracle_grid_cells(const or_particle* atoms, int n_atoms, const double t[9], const int rep[3],
                      double rc2, int nx, int ny, int nz, double* energy, double* sum_abs,
                      int n_threads);
/* oracle_henry with the cell-list energy (same points, mask test and output). */
int oracle_henry_cells(const or_particle* atoms, int n_atoms, const double t[9],
                       const int rep[3], double rc2, double T, uint64_t seed, int64_t n_ins,
                       const uint8_t* mask, int mnx, int mny, int mnz, double* out,
                       double* energies, int n_threads);

/* ---- er_oracle_synth.c: the benchmark's seeded frameworks ---- */
int oracle_cell_matrices(double a, double b, double c, double alpha_deg, double beta_deg,
                         double gamma_deg, double t[9], double inv[9], double* volume);
int oracle_replication_factors(const double t[9], double r_cutoff, int factor, int rep[3]);
int oracle_synth_positions(uint64_t seed, const double t[9], int n_atoms, double d_min,
                           double* frac);

#ifdef __cplusplus
}
#endif

#endif /* ER_ORACLE_H_ */
