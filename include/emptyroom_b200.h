/*
 * emptyroom_b200.h -- C ABI of the B200 (sm_100a) adsorption hot path.
 *
 * One shared library, libemptyroom_b200.so, replaces the device-compute seam of
 * CorySimon/EmptyRoom: the kernel launches in src/writegrid.cu and src/henry.cu
 * and the CPU flood fill of src/pocketblocking.cc. Signatures use plain C
 * types only. Every call returns an er_status (ER_OK == 0) and never exits the
 * process; er_ctx_last_error() describes the last failure of a context.
 * A context is used by one host thread at a time; contexts are independent.
 * Host buffers stay owned by the caller.
 */
#ifndef EMPTYROOM_B200_H_
#define EMPTYROOM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    ER_OK = 0,
    ER_ERR_INVALID = 1,   /* bad argument (sizes, ids, NULL) */
    ER_ERR_CUDA = 2,      /* CUDA runtime error or no usable device */
    ER_ERR_NOMEM = 3,     /* device or host allocation failed / over budget */
    ER_ERR_IO = 4,        /* file could not be read or written */
    ER_ERR_NOT_FOUND = 5, /* label / id not found */
    ER_ERR_TIMEOUT = 6,   /* a bounded wait ran out */
    ER_ERR_LIMIT = 7      /* a documented size limit was exceeded */
} er_status;

const char* er_status_string(int status);

/* ------------------------------------------------------------------ types */
/* Same field order and meaning as FrameworkParticle (src/datatypes.h:20-28):
 * fractional position and the Lorentz-Berthelot mixed epsilon (K) and
 * sigma^2 (A^2) of this framework atom with the probe. */
typedef struct {
    double x_f, y_f, z_f;
    double eps_with_adsorbate;
    double sig_with_adsorbate_squared;
} er_particle;

/* What the reference passes to its kernels by value in GridParameters /
 * HenryParameters (src/datatypes.h:44-110): the atoms, the fractional ->
 * Cartesian matrix (row-major, src/Framework.cc:124-132), the unit-cell
 * replication factors (images -rep..rep per axis) and the squared cutoff. */
typedef struct {
    int n_atoms;
    const er_particle* atoms; /* host pointer, n_atoms entries */
    double t_matrix[9];
    int rep[3];
    double r_cutoff_squared;
} er_framework_desc;

typedef struct er_ctx er_ctx;

/* ------------------------------------------------------------------ context */
/* Binds `device`, creates the context's stream and allocator. */
int er_ctx_create(int device, er_ctx** out);
void er_ctx_destroy(er_ctx* ctx);
const char* er_ctx_last_error(const er_ctx* ctx);
/* Waits for all work queued on the context's stream. */
int er_ctx_synchronize(er_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against the library's launches. */
int er_ctx_stream(er_ctx* ctx, void** stream);

/* ------------------------------------------------------------------ frameworks */
/* Uploads a framework/probe pair and builds its device-resident image cell
 * list (on the host, then copied). Replaces the cudaMalloc/cudaMemcpy of
 * FrameworkParticle[] at src/writegrid.cu:187-189 and src/henry.cu:133-135.
 * *fw_id receives a handle. */
int er_framework_upload(er_ctx* ctx, const er_framework_desc* desc, int* fw_id);
/* Uploads n frameworks at once: only the atoms are copied (56 bytes each),
 * and the image cell lists are built on the device, equal bit for bit to
 * er_framework_upload's. Validation runs on the host first, with the same
 * errors; on error no handle is created. (No counterpart in the reference,
 * which reads one framework per process.) */
int er_framework_upload_many(er_ctx* ctx, const er_framework_desc* descs, int n, int* fw_ids);
int er_framework_release(er_ctx* ctx, int fw_id);
/* Device bytes held by a framework handle. */
int er_framework_bytes(er_ctx* ctx, int fw_id, size_t* bytes);

/* ------------------------------------------------------------------ grids */
/* Output placement / type / precision flags for er_grid. */
#define ER_OUT_HOST 0x0      /* out is a host pointer (copied back inside the call) */
#define ER_OUT_DEVICE 0x1    /* out is a device pointer on the context's device */
#define ER_OUT_F32 0x0       /* float per point */
#define ER_OUT_F64 0x2       /* double per point (the reference's sheet type) */
#define ER_PREC_NEAR64 0x0  /* default: FP32 pair terms except the pairs of atoms within
                                5 A of a warp's points, which are FP64 (the large terms
                                whose FP32 rounding dominates where terms cancel); FP32
                                sums of 16 terms (64 on the cutoff shell) folded into
                                FP64 per-point totals. Within 1e-5 relative of FP64 on
                                points with E < -10 K */
#define ER_PREC_COMP 0x08    /* all pair terms FP32, FP32 sums of 64 terms folded into
                                FP64 per-point totals: faster, but its error on E < 0
                                points reaches ~2e-5 relative where large near terms
                                cancel */
#define ER_PREC_FP32 0x10    /* FP32 pair terms, plain FP32 accumulation */
#define ER_PREC_FP64 0x20    /* FP64 pair terms and accumulation, same pair set as the
                                FP32 modes (precision sweeps); needs ER_OUT_F64 */
#define ER_COUNT_PAIRS 0x40  /* diagnostic: write the number of in-cutoff pair terms per
                                point instead of the energy (same traversal) */
#define ER_TILE_P8 0x80      /* kernel variant with 8 points per thread (16 x 8 x 16
                                bricks) instead of 4; results agree within the FP32
                                tolerance, not bit for bit */

/* Energies above this value (K) are written as this value (overflow cap). */
#define ER_ENERGY_CAP 1.0e30

/* Probe-framework LJ energy (K) at every point of an nx x ny x nz grid with
 * fractional axes i/(N-1), endpoints included, layout out[k + j*nz + i*ny*nz]:
 * the values ComputeGridSheet (src/computegridsheet.h:30-99) produces for all
 * x-sheets of src/writegrid.cu:219-226. Requires nx, ny, nz >= 2. */
int er_grid(er_ctx* ctx, int fw_id, int nx, int ny, int nz, int flags, void* out);

/* One x = x_index sheet as double[ny*nz] on the host, index k + j*nz: the
 * drop-in for one ComputeGridSheet launch plus its D2H copy
 * (src/writegrid.cu:221-232). */
int er_grid_sheet(er_ctx* ctx, int fw_id, int nx, int ny, int nz, int x_index,
                  double* out_sheet);

/* Hard-sphere accessibility (1 accessible, 0 overlap: some image within
 * +-1 cells has r^2 < sigma_mix^2), the ComputeGridSheetAccessibleOrNot
 * semantics of src/computegridsheet.h:101-165, host uint8 out. */
int er_accessibility(er_ctx* ctx, int fw_id, int nx, int ny, int nz, uint8_t* out);

/* ------------------------------------------------------------------ batches */
typedef struct {
    int fw_id;
    int nx, ny, nz;
    float* out_device; /* device buffer of nx*ny*nz floats */
} er_grid_job;

#define ER_BATCH_PERSISTENT 0 /* one persistent launch over a device work queue */
#define ER_BATCH_PLAIN 1      /* one plain launch per job, in order */
#define ER_BATCH_HOST_OUT 0x100 /* or-ed into mode: out_device fields are host pointers;
                                   grids are staged on the device and copied back */
#define ER_BATCH_AUTOTUNE 0x200 /* or-ed into mode: pick each job's kernel variant (4 or
                                   8 points per thread) by timing both on a sample of the
                                   first job of its class (atom density, grid spacing,
                                   cutoff); choices are cached in the context. A job's
                                   result then equals er_grid with that variant's flag. */
#define ER_BATCH_COMP 0x400 /* or-ed into mode: the ER_PREC_COMP pair sum (all pair terms
                               FP32) instead of the default ER_PREC_NEAR64; results then
                               equal er_grid with ER_PREC_COMP */

/* Runs many grid jobs (uneven frameworks, probes, grid sizes). Results are
 * identical between the two modes and independent of the job mix; each job
 * equals er_grid of the same framework and dims with the same precision flag
 * (and ER_TILE_P8 where the plan picked that variant). */
int er_grid_batch(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode);

/* A batch plan fixes the work queue once and replays it as a CUDA graph. */
typedef struct er_batch_plan er_batch_plan;
int er_batch_plan_create(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode,
                         er_batch_plan** out);
int er_batch_plan_run(er_batch_plan* plan); /* asynchronous on the context stream */
/* Kernel launches one run of the plan issues (its CUDA graph's kernel nodes). */
int er_batch_plan_launches(const er_batch_plan* plan, int* n_launches);
/* Points per thread (4 or 8) of the kernel variant the plan uses for job `job`
 * (8: reproduce with ER_TILE_P8 in er_grid). */
int er_batch_plan_tile(const er_batch_plan* plan, int job, int* tile_p);
void er_batch_plan_destroy(er_batch_plan* plan);

/* ------------------------------------------------------------------ Widom / Henry */
typedef struct {
    double sum_w;           /* sum over insertions of exp(-E/T) */
    double sum_ew;          /* sum of E exp(-E/T) (K) */
    double log_scale;       /* m: sum_w = sum_w_scaled * exp(m) (log-sum-exp form) */
    double sum_w_scaled;    /* sum of exp(-E/T - m) */
    double sum_ew_scaled;   /* sum of E exp(-E/T - m) */
    double n_insertions;    /* insertions performed (blocked ones included) */
    double n_blocked;       /* insertions that fell in a blocked grid cell */
    double mean_energy;     /* <E> = sum_ew / sum_w (K) */
    double kh_mol_m3_pa;    /* K_H = sum_w / (N T 8.314), src/henry.cu:169 */
} er_henry_result;

/* Widom insertions i = 0..n_ins-1 at Philox4x32-10 points of stream `seed`
 * (fractional coordinates uniform in [0,1), 53 bits each), E by the pair sum
 * of src/doHenry.h:70-98, FP64 log-sum-exp reduction of
 * src/doHenry.h:106-125 and src/henry.cu:157-169. block_mask (host or device
 * memory, may be NULL) is an mnx x mny x mnz grid (axes i/(N-1)), e.g. the
 * pocket mask of er_block_pockets_device; an insertion whose 8 surrounding
 * corners include a set entry is blocked and has weight 0.
 * energies_out (host, may be NULL) receives E per insertion as float. */
int er_henry(er_ctx* ctx, int fw_id, double temperature, int64_t n_ins, uint64_t seed,
             const uint8_t* block_mask, int mnx, int mny, int mnz, er_henry_result* out,
             float* energies_out);

/* Widom insertions for n frameworks: the henry tool's per-structure run
 * (src/henry.cu:63-174, one structure per process there) for many structures
 * in one call. For entry k: when the blocking dims are non-zero (each >= 2),
 * the FP32 energy grid of block_nx x block_ny x block_nz points (as er_grid
 * with default flags), its pocket mask (as er_block_pockets_device, pocketblocking.cc:
 * 126-391) and er_henry of fw_ids[k] with seed seeds[k] and that mask; with
 * all three dims 0, er_henry alone. The frameworks run on up to six
 * concurrent pipelines (a stream, scratch and a host thread each, kept by the
 * context; fewer when half the free device memory holds fewer pipelines'
 * scratch, about 40 bytes per insertion and 24 per blocking-grid point each),
 * so that one framework's grid, labelling, binning and host round trips
 * overlap another's energy kernel. Each results[k] (and n_pockets[k],
 * when n_pockets is not NULL) equals the single calls' bit for bit. On an
 * error the remaining entries are not run. */
int er_henry_batch(er_ctx* ctx, const int* fw_ids, int n, double temperature,
                   int64_t n_insertions, const uint64_t* seeds, int block_nx, int block_ny,
                   int block_nz, er_henry_result* results, int* n_pockets);

/* Device time (ms) of each stage of the last er_henry call on ctx, taken with
 * CUDA events on the context stream while timing is on (er_ctx_set_timing,
 * off by default): Philox points, mask test and bin counts; the bin layout
 * (scatter into bins, placement of each point, ordering of the bins that
 * straddle a warp boundary); the Lennard-Jones energy kernel; the FP64
 * log-sum-exp reduction. The reference
 * times only the whole run ("Simulation time", src/henry.cu:150-153).
 * er_henry_batch, the server and er_henry_stats_noalloc record nothing. */
typedef struct {
    double bin_ms, sort_ms, energy_ms, reduce_ms;
} er_henry_timing;
int er_ctx_set_timing(er_ctx* ctx, int on);
int er_henry_last_timing(er_ctx* ctx, er_henry_timing* out);

/* Widom statistics of energies the caller already holds on the device,
 * computed without allocating anything: no counterpart in the reference.
 * For callers that cannot call cudaMalloc -- a code that reserves all of its
 * device memory up front in its own pool, or a loop that cannot take the
 * implicit synchronisation and unbounded latency of cudaMalloc/cudaFree.
 * energies: device float[n]. An entry of +inf has weight 0 and is counted in
 * n_blocked; a NaN or -inf entry has no defined weight and makes the call
 * return ER_ERR_INVALID. The result is er_henry's reduction (FP64
 * log-sum-exp, the same block partition) with n_insertions = n. Its scratch
 * is one file-scope static device array of 4097 x 40 bytes, held by every GPU
 * that loads this library until the process exits. The first call on a
 * device looks up that array's address (cudaGetSymbolAddress) with the
 * device current; make that first call before any stream capture begins.
 * The call is synchronous: it returns once the result has reached the host.
 * Calls that overlap on one GPU (from several host threads or contexts)
 * share the array and race. n outside [1, ER_HENRY_STATS_NOALLOC_MAX_N] is
 * rejected with ER_ERR_LIMIT. */
#define ER_HENRY_STATS_NOALLOC_MAX_N 2147483647LL
int er_henry_stats_noalloc(er_ctx* ctx, const float* energies, int64_t n, double temperature,
                           er_henry_result* out);

/* ------------------------------------------------------------------ pocket blocking */
/* FindAndBlockPockets (src/pocketblocking.cc:126-391) on the GPU: points with
 * E >= 15 T are inaccessible; accessible points form 6-connected segments
 * (no periodic wrap); segments linked across the periodic faces are
 * classified CHANNEL or POCKET; pocket points are overwritten with 1e13.
 * grid is a host double[nx*ny*nz] modified in place; *n_pockets receives the
 * reference's return value. segments_out (host, may be NULL) receives the
 * segment id per point (-1 inaccessible) in the reference's numbering. */
int er_block_pockets(er_ctx* ctx, double* grid, int nx, int ny, int nz, double temperature,
                     int* n_pockets, int* segments_out);

/* Device form: grid is a device float[nx*ny*nz] (left unchanged);
 * pocket_mask_out (device uint8[nx*ny*nz]) receives 1 at pocket points. */
int er_block_pockets_device(er_ctx* ctx, const float* grid, int nx, int ny, int nz,
                            double temperature, uint8_t* pocket_mask_out, int* n_pockets);

/* ------------------------------------------------------------------ GCMC lookup */
/* Guest-framework energies of a GCMC code by trilinear interpolation of a
 * device-resident grid: out[q] = GuestFrameworkEnergy(WrapToInterval(x, 1),
 * WrapToInterval(y, 1), WrapToInterval(z, 1)) of src/gcmc.cc:145-177 and
 * :74-77 at pts[3q..3q+2] (fractional), FP64 arithmetic in the reference's
 * order, so equal bit for bit to the reference function on the same grid
 * values. grid: device memory, nx*ny*nz, layout k + j nz + i ny nz, float
 * (as er_grid writes it) or double with ER_INTERP_GRID_F64. pts / out: host
 * or device memory. The lower corner index is clamped to N - 2 (the reference
 * reads past the grid when x / dx rounds up to N - 1 for x just below 1). */
#define ER_INTERP_GRID_F64 0x1
int er_grid_interp(er_ctx* ctx, const void* grid, int nx, int ny, int nz, int flags,
                   const double* pts, int64_t n, double* out);

/* ------------------------------------------------------------------ host helpers */
/* Fractional -> Cartesian matrix and its inverse from cell lengths (A) and
 * angles (degrees), the formulas of src/Framework.cc:113-142. Returns
 * ER_ERR_INVALID for a degenerate cell. volume receives V (A^3). */
int er_cell_matrices(double a, double b, double c, double alpha_deg, double beta_deg,
                     double gamma_deg, double t_matrix[9], double inv_t_matrix[9],
                     double* volume);

/* Replication factors floor(rc / w_i) + 1, w_i the perpendicular cell widths:
 * enough images that every image within rc of any grid point is summed
 * (the .uc files read at src/readsettings.h:243-274). factor 2 gives the
 * "twice" variant (w_i >= 2 rc per replicated cell). */
int er_replication_factors(const double t_matrix[9], double r_cutoff, int factor, int rep[3]);

/* Philox4x32-10 block (host copy of the device generator). */
void er_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Insertion point i of stream seed (the points er_henry uses). */
void er_insertion_point(uint64_t seed, uint64_t i, double out[3]);

/* Seeded synthetic framework: n_atoms fractional positions uniform in [0,1)
 * with minimum periodic pair distance d_min (A, 0 disables), rejection
 * sampled with a cell list. Returns ER_ERR_LIMIT when the density cannot
 * be reached within the attempt budget. */
int er_synth_positions(uint64_t seed, const double t_matrix[9], int n_atoms, double d_min,
                       double* frac_out);

/* ------------------------------------------------------------------ serving */
/* A request server over one context: jobs are submitted from any host thread
 * as they arrive; a scheduler thread admits them while a job slot is free and
 * their device footprint fits the HBM budget, and launches each admitted job
 * on its slot's stream, so jobs that arrive while others run execute
 * concurrently on the device (continuous batching). Admission is size-aware:
 * jobs cheaper than the running median (points x atom density) go to slots
 * created at the highest stream priority, others to low-priority slots; the
 * oldest job is overtaken by none once it has waited 50 ms. Framework images
 * and finished grids stay resident on the device (caches keyed by the
 * caller's framework key and the grid size); least recently used grids are
 * evicted when the budget needs room; with the budget full, a new grid takes
 * over the buffer of an idle grid that holds it (at most twice its size)
 * before any grid memory goes back to the pool. A job's result does not
 * depend on which other jobs run beside it. With slots = 1 the server runs one
 * job at a time (the plain one-job-per-launch loop). The reference has no
 * serving layer. er_server_create reserves the budget in the context's memory
 * pool and each slot's Widom scratch (an eighth of the budget over all slots,
 * at most 2^24 insertions per slot; it counts against the budget). While a
 * server exists its scheduler thread uses the context: make no other calls on
 * that context, and destroy the server before the context. */
typedef struct er_server er_server;
#define ER_JOB_GRID 1
#define ER_JOB_HENRY 2
typedef struct {
    int kind;                        /* ER_JOB_GRID or ER_JOB_HENRY */
    uint64_t fw_key;                 /* caller's key of the framework/probe pair */
    const er_framework_desc* desc;   /* read (host) when fw_key is not resident yet;
                                        must stay valid until the job completes */
    int nx, ny, nz;                  /* grid jobs */
    double temperature;              /* Henry jobs */
    int64_t n_insertions;
    uint64_t seed;
    float* grid_out_host;            /* optional host copy of the grid (pinned memory
                                        keeps the copy asynchronous) */
} er_job;
typedef struct {
    int done;                        /* 1 once finished (status holds the outcome) */
    int status;                      /* er_status of the job */
    int grid_cache_hit;              /* the grid was already resident */
    double submit_s, start_s, finish_s; /* server clock, seconds */
    er_henry_result henry;           /* Henry jobs */
} er_job_status;
int er_server_create(er_ctx* ctx, size_t hbm_budget_bytes, int slots, er_server** out);
/* Thread-safe; returns at once with a ticket (>= 1). */
int er_server_submit(er_server* s, const er_job* job, uint64_t* ticket);
/* Copies the job's status; ER_ERR_NOT_FOUND for an unknown ticket. */
int er_server_poll(er_server* s, uint64_t ticket, er_job_status* st);
/* Waits up to timeout_s for the job; ER_ERR_TIMEOUT when it is still running. */
int er_server_wait(er_server* s, uint64_t ticket, double timeout_s, er_job_status* st);
/* Device pointer of a finished grid job's resident grid, valid until that
 * grid is evicted or the server is destroyed. Once the budget is full, an
 * evicted grid's buffer may be taken over by a later grid job and hold
 * another framework's grid: a caller that keeps using the pointer must not
 * submit grid jobs in the meantime, and orders its own reads (on its own
 * streams) itself, since only server jobs pin a grid. */
int er_server_grid(er_server* s, uint64_t ticket, const float** grid);
/* Server clock (seconds), the clock of er_job_status. */
double er_server_now(const er_server* s);
/* Device bytes held by resident frameworks, grids and job scratch. */
int er_server_bytes(const er_server* s, size_t* bytes);
/* Drains running jobs and frees everything the server holds. */
void er_server_destroy(er_server* s);

/* ------------------------------------------------------------------ file formats */
/* The reference's input files, read the way its loaders read them. Paths are
 * relative to `root` (the reference runs from its project root). Errors are
 * returned (ER_ERR_IO / ER_ERR_NOT_FOUND / ER_ERR_INVALID) with a message in
 * err[0..errlen), never exit(). */

/* A parsed .cssr structure: Framework(name) of src/Framework.cc:13-178 --
 * <root>/data/structures/<name>.cssr (a b c; alpha beta gamma in degrees;
 * atom count; a skipped title line; atom lines `idx label x_f y_f z_f ...`
 * with coordinates wrapped by fmod(x, 1.0)) and masses from
 * <root>/data/masses.def. */
typedef struct er_structure er_structure;
int er_structure_load(const char* root, const char* name, er_structure** out, char* err,
                      size_t errlen);
void er_structure_free(er_structure* s);
/* cell[6] = a, b, c (A), alpha, beta, gamma (radians, as Framework stores them);
 * t and inv row-major; volume (A^3); density (kg/m^3). */
int er_structure_info(const er_structure* s, int* n_atoms, double cell[6], double t[9],
                      double inv[9], double* volume, double* density);
/* frac: n_atoms x 3 (after fmod). */
int er_structure_frac(const er_structure* s, double* frac);
/* Label of atom i into buf (NUL-terminated). */
int er_structure_label(const er_structure* s, int i, char* buf, size_t len);

/* A force field: Forcefield(name) of src/Forcefield.cc:15-54 --
 * <root>/data/forcefields/<name>.def, first line skipped, lines `label eps sigma`. */
typedef struct er_forcefield er_forcefield;
int er_forcefield_load(const char* root, const char* name, er_forcefield** out, char* err,
                       size_t errlen);
void er_forcefield_free(er_forcefield* f);
int er_forcefield_count(const er_forcefield* f);
int er_forcefield_entry(const er_forcefield* f, int i, char* label, size_t len, double* eps,
                        double* sig);
/* First entry with this label (GrabGuestForceFieldParams, src/readsettings.h:276-294). */
int er_forcefield_find(const er_forcefield* f, const char* label, double* eps, double* sig);

/* FrameworkParticle array with Lorentz-Berthelot mixing against the guest:
 * LoadFastFrameworkParticleArray, src/load_fast_particle_f_array.h:13-40.
 * out holds n_atoms entries. ER_ERR_NOT_FOUND names the first missing label. */
int er_mix_particles(const er_structure* s, const er_forcefield* f, double eps_guest,
                     double sig_guest, er_particle* out, char* err, size_t errlen);

/* Adsorbate molecular weight from <root>/data/masses.def (GetAdsorbateMW,
 * src/readsettings.h:19-49). */
int er_adsorbate_mw(const char* root, const char* adsorbate, double* mw, char* err,
                    size_t errlen);

/* Replication factors from <root>/data/uc_replications/<name>_<which>.uc
 * (ReadUnitCellReplicationFile, src/readsettings.h:243-274). */
int er_read_uc(const char* root, const char* name, const char* which, int rep[3], char* err,
               size_t errlen);
/* Writes the .uc file with er_replication_factors(t, rc, factor). */
int er_write_uc(const char* root, const char* name, const char* which, const int rep[3]);

/* simulation.input keys (src/readsettings.h:51-156): token scan, unknown words
 * ignored, defaults as the reference's. */
typedef struct {
    char forcefield[256];       /* "None" when absent */
    int verbose;
    double grid_resolution;     /* -1 when absent */
    char grid_output_format[16];/* "txt" default */
    double r_cutoff_squared;    /* 12.5^2 default */
    int feynman_hibbs;
    double energy_threshold;
    double temperature;         /* -1 when absent */
    int insertions_per_a3;      /* -1 when absent */
} er_settings;
#define ER_SETTINGS_GRID 1
#define ER_SETTINGS_HENRY 2
/* Reads <path> and checks the keys the given tool requires (same checks and
 * messages as the reference). */
int er_read_settings(const char* path, int kind, er_settings* out, char* err, size_t errlen);

/* Grid text file of src/writegrid.cu:142-147,260-269: header
 * "%d %d %d  = (N_x,N_y,N_z) grid points (grid is in fractional coords). Endpoints included.\n"
 * then one line per (x, y) pencil of N_z values "% 13.6E ". Values are printed
 * from double(grid[k + j nz + i ny nz]). Formatting is split over n_threads
 * host threads (0 = all cores); bytes are identical to a serial fprintf. */
int er_write_grid_txt(const char* path, const float* grid, int nx, int ny, int nz,
                      int n_threads);
/* .cube variant of src/writegrid.cu:149-166,244-258: header from t, values in
 * kJ/mol (x 8.314 / 1000), six per line, newline after each pencil. */
int er_write_grid_cube(const char* path, const float* grid, int nx, int ny, int nz,
                       const double t[9], int n_threads);
/* Reader with the layout contract of src/gcmc.cc:293-345: fills out (capacity
 * `cap` doubles, index k + j nz + i ny nz) and dims. */
int er_read_grid_txt(const char* path, double* out, size_t cap, int dims[3], char* err,
                     size_t errlen);

/* ------------------------------------------------------------------ diagnostics */
/* Measures the device's FP32 FMA issue rate with a chain of independent FFMAs
 * (FP32-pipe lane-instructions per second, whole GPU) over about `seconds`.
 * This is the denominator of the pair-sum roofline. */
int er_probe_fp32_rate(er_ctx* ctx, double seconds, double* instr_per_s);

/* Largest relative error |1 - x y0| of the hardware FP64 reciprocal seed y0
 * (rcp.approx.ftz.f64) over ~2e7 squared distances x in [2^-80, 2^20): the
 * seed the near pairs of ER_PREC_NEAR64 refine by one Newton step, whose
 * error is the square of this. No counterpart in the reference (FP64 `/`). */
int er_probe_rcp64_seed(er_ctx* ctx, double* max_rel_err);

/* Self-test of the kernels' bounded waits: one CTA waits, `spins` polls at
 * most, for a completion barrier that nothing completes; the wait must give
 * up, raise the context's fault word and let the host see it (ER_OK then;
 * ER_ERR_CUDA if it did not report). The context stays usable. The staged
 * producer (build option ER_BULK=1) waits the same way with 2^22 polls. No
 * counterpart in the reference. */
int er_selftest_wait_timeout(er_ctx* ctx, int spins);

/* Library version string. */
const char* er_version(void);

#ifdef __cplusplus
}
#endif

#endif /* EMPTYROOM_B200_H_ */
