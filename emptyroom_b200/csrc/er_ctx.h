// er_ctx.h -- the context object behind the C ABI (host side only).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <thread>
#include <tuple>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/emptyroom_b200.h"
#include "er_internal.h"

namespace er {

// One uploaded framework: a single device allocation holding every array.
struct FwRecord {
    FwDev dev{};
    void* block = nullptr;
    size_t bytes = 0;
    double rc2 = 0.0;
    double t[9] = {0};
    double cell_len[3] = {0, 0, 0};  // |a|, |b|, |c|
    double volume = 0.0;
    int n_atoms = 0;
};

// A grow-only device buffer.
struct DevBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    cudaStream_t owner = nullptr;  // stream-ordered buffers: the stream they live on
    int ensure(size_t bytes);
    // Grows from `pool` in stream order on `st` (the old buffer is freed on
    // `st` too): no device-wide synchronisation, for buffers one stream uses.
    int ensure_on(size_t bytes, cudaMemPool_t pool, cudaStream_t st);
    void release();
};

// A grow-only pinned host buffer.
struct HostBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
};

// Device scratch of one Widom pipeline (er_henry.cu); one per stream that
// runs Widom jobs concurrently.
struct HenryScratch {
    DevBuf pts, bin, order, tmp, counts, starts, e, nblk, part, res, mask, cell;
    // stage boundaries of the last run (er_ctx_set_timing): start, binned,
    // sorted, energies, reduced; ev[0] == nullptr while timing is off
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t bytes() const {
        return pts.cap + bin.cap + order.cap + tmp.cap + counts.cap + starts.cap + e.cap +
               nblk.cap + part.cap + res.cap + mask.cap + cell.cap;
    }
    void release() {
        DevBuf* b[] = {&pts, &bin, &order, &tmp, &counts, &starts, &e, &nblk, &part, &res, &mask,
                       &cell};
        for (DevBuf* x : b) x->release();
    }
};

// Host copy of a Widom reduction: (m, s, se) and the blocked count.
struct HenryOut {
    double lse[3];
    int n_blocked;
};

// Device scratch of one pocket-blocking run (er_pockets.cu): labels,
// segments, per-segment flags, scan/link tables, a grid copy, the FP64 grid
// of er_block_pockets.
struct PocketScratch {
    DevBuf grid, lab, seg, flags, misc, mask;
    void release() {
        DevBuf* b[] = {&grid, &lab, &seg, &flags, &misc, &mask};
        for (DevBuf* x : b) x->release();
    }
};

// One pipeline of er_henry_batch: its stream and everything a framework's
// grid -> pocket mask -> Widom run needs, so that pipelines overlap.
struct HenryPipe {
    cudaStream_t stream = nullptr;
    HenryScratch hs;
    PocketScratch ps;
    DevBuf grid, mask;
    HenryOut* out = nullptr;  // pinned
};

}  // namespace er

struct er_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // device->host copies overlapping the kernels
    std::string last_error;
    std::map<int, er::FwRecord> fws;
    int next_fw = 1;
    double cell_edge = 2.0;  // cell-list edge (A)
    std::map<std::tuple<int, int, int, int>, int> tune;  // autotuned kernel variant per job class
    // scratch
    er::DevBuf grid_f32;     // staging for host-bound grids
    er::DevBuf counter;      // scratch of the FP32 rate probe
    er::HostBuf pinned;      // pinned staging
    er::HostBuf plan_pinned; // pinned staging of batch-plan queues
    cudaMemPool_t pool = nullptr;  // stream-ordered pool (framework blocks, plan queues)
    er::DevBuf task_left;    // per-job bricks left (completion notification)
    int* fault_host = nullptr;  // mapped pinned word a kernel sets when a bounded wait
    int* fault_dev = nullptr;   // gives up (FwDev::fault of every framework), its device address
    int* done_host = nullptr;   // mapped pinned per-job completion flags
    int* done_dev = nullptr;    // the same flags, device address
    size_t done_cap = 0;
    // Widom scratch
    er::HenryScratch henry;
    // pocket-blocking scratch
    er::PocketScratch pocket;
    // pipelines of er_henry_batch (created on first use)
    std::vector<er::HenryPipe*> pipes;
    std::mutex err_mu;  // last_error is written by er_henry_batch's workers too
    // staging of host points / results for er_grid_interp
    er::DevBuf interp;
    // device-resident grid cache for er_grid_sheet: key (fw, nx, ny, nz)
    struct SheetCache {
        int fw = 0, nx = 0, ny = 0, nz = 0;
        er::DevBuf grid;
    } sheet_cache;
};

namespace er {

struct HostFramework;

// Byte layout of one framework's device block (every array 256-byte aligned):
// images (double4), (C12, -C6) (float2), image ids (u32), cell_start
// (ncell + 1 ints), atom_frac (double4), atom_lj64 (double2), and the FP64
// (C12, C6) of every image (double2, the near pairs of the NEAR64 mode).
struct FwLayout {
    size_t o_par, o_id, o_cs, o_af, o_lj, o_ilj, total;
};
FwLayout fw_layout(size_t n_img, size_t n_cs, size_t n_atoms);
// Fills the handle record of a framework whose block is (being) written at `block`.
void fw_record(const HostFramework& hf, size_t n_img, const FwLayout& L, void* block,
               FwRecord& rec);
// Uploads with the image cell lists built on the host threads.
int host_upload_many(er_ctx* ctx, const er_framework_desc* descs, int n, int* fw_ids);

// Runs f(i) for i in [0, n) on up to hardware_concurrency host threads.
template <class F>
void parallel_for(int n, F&& f) {
    const int nt = std::max(1, std::min<int>(n, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next(0);
    auto worker = [&]() {
        for (int i; (i = next.fetch_add(1)) < n;) f(i);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(worker);
    worker();
    for (auto& x : th) x.join();
}

int set_error(er_ctx* ctx, int status, const std::string& msg);
// Device memory from the context's pool, ordered on ctx->stream; the pool
// keeps freed memory for reuse (trimmed and retried once when exhausted).
int pool_alloc(er_ctx* ctx, void** p, size_t bytes);
int cuda_error(er_ctx* ctx, cudaError_t e, const char* what);
// ER_ERR_CUDA (and the word cleared) when a kernel has set the context's
// fault word since the last check, else ER_OK.
int take_fault(er_ctx* ctx);
const FwRecord* find_fw(er_ctx* ctx, int fw_id);
// Cutoff constants for a framework and a CTA box diagonal (A).
CutoffConsts make_cutoff_consts(double rc2, double box_diag, double r2min);
// Grid dimensions accepted by every grid entry point: each >= 2 (axes
// i / (N - 1)) and at most 4e9 points; checked before any allocation.
int check_grid_dims(er_ctx* ctx, int nx, int ny, int nz, const char* who);
// Fills a grid task (validates dims) and launches the plain grid kernel on `st`.
int fill_grid_task(er_ctx* ctx, const FwRecord& fw, int nx, int ny, int nz, float* out,
                   GridTask& t, int tile_p = 4);
int launch_grid_plain_on(er_ctx* ctx, const GridTask& t, int prec, cudaStream_t st);
// Widom pipeline on stream `st` with scratch `hs`; when host_out (pinned) is
// given, the reduction and the blocked count are copied there asynchronously.
int henry_check(er_ctx* ctx, double temperature, int64_t n_ins, const uint8_t* block_mask,
                int mnx, int mny, int mnz);
// Grows the per-insertion scratch of `hs` to hold n insertions (stream order).
int henry_reserve(er_ctx* ctx, HenryScratch& hs, int64_t n, cudaStream_t st);
int henry_enqueue(er_ctx* ctx, const FwRecord& fw, double temperature, int n, uint64_t seed,
                  const uint8_t* block_mask, int mnx, int mny, int mnz, cudaStream_t st,
                  HenryScratch& hs, HenryOut* host_out);
void henry_finish(const HenryOut& h, int64_t n, double temperature, er_henry_result* out);
// Pocket mask of an FP32 device grid (er_block_pockets_device) with scratch
// `ps` on stream `st`; synchronises `st` (the segment classification runs on
// the host).
int block_pockets_device_on(er_ctx* ctx, PocketScratch& ps, cudaStream_t st, const float* grid,
                            int nx, int ny, int nz, double temperature, uint8_t* mask_out,
                            int* n_pockets);
// Exclusive scan of n ints on `st`: out[0..n] (out[n] = the total), with
// scan_tiles(n) ints of scratch in tile_sums.
int scan_tiles(int n);
int scan_exclusive(er_ctx* ctx, const int* in, int n, int* out, int* tile_sums, cudaStream_t st);
// Builds the image cell lists of n frameworks on the device (er_build.cu).
int device_upload_many(er_ctx* ctx, const er_framework_desc* descs, int n, int* fw_ids);

}  // namespace er

#define ER_CUDA(ctx, call)                                      \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return er::cuda_error(ctx, _e, #call); \
    } while (0)

// Synchronises `stream`, then reports a fault a kernel raised in the
// context's fault word (a bounded wait that gave up) as ER_ERR_CUDA.
#define ER_SYNC(ctx, stream)                                    \
    do {                                                        \
        ER_CUDA(ctx, cudaStreamSynchronize(stream));            \
        if (int _f = er::take_fault(ctx)) return _f;            \
    } while (0)
