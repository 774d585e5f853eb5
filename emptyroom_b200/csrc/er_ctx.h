// er_ctx.h -- the context object behind the C ABI (host side only).
#pragma once
#include <cuda_runtime.h>

#include <map>
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
    int ensure(size_t bytes);
    void release();
};

// A grow-only pinned host buffer.
struct HostBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes);
    void release();
};

}  // namespace er

struct er_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    std::map<int, er::FwRecord> fws;
    int next_fw = 1;
    double cell_edge = 2.0;  // cell-list edge (A)
    // scratch
    er::DevBuf grid_f32;     // staging for host-bound grids
    er::DevBuf tasks;        // GridTask arrays for batches
    er::DevBuf items;        // WorkItem queues
    er::DevBuf counter;      // persistent-queue heads
    er::HostBuf pinned;      // pinned staging
    // Widom scratch
    er::DevBuf h_pts, h_bin, h_order, h_tmp, h_counts, h_starts, h_wt, h_nwt, h_e, h_part,
        h_mask, h_res;
    // pocket-blocking scratch
    er::DevBuf p_grid, p_lab, p_seg, p_flags, p_misc, p_mask;
    // device-resident grid cache for er_grid_sheet: key (fw, nx, ny, nz)
    struct SheetCache {
        int fw = 0, nx = 0, ny = 0, nz = 0;
        er::DevBuf grid;
    } sheet_cache;
};

namespace er {

int set_error(er_ctx* ctx, int status, const std::string& msg);
int cuda_error(er_ctx* ctx, cudaError_t e, const char* what);
const FwRecord* find_fw(er_ctx* ctx, int fw_id);
// Cutoff constants for a framework and a CTA box diagonal (A).
CutoffConsts make_cutoff_consts(double rc2, double box_diag, double r2min);

}  // namespace er

#define ER_CUDA(ctx, call)                                      \
    do {                                                        \
        cudaError_t _e = (call);                                \
        if (_e != cudaSuccess) return er::cuda_error(ctx, _e, #call); \
    } while (0)
