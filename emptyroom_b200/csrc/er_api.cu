// er_api.cu -- context, framework upload and the grid entry points of the C ABI.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "er_ctx.h"
#include "er_engine.cuh"
#include "er_host.h"

namespace er {

int DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && ptr) return ER_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    if (cudaMalloc(&ptr, want) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return ER_ERR_NOMEM;
    }
    cap = want;
    return ER_OK;
}
void DevBuf::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}
int HostBuf::ensure(size_t bytes) {
    if (bytes <= cap && ptr) return ER_OK;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    if (cudaMallocHost(&ptr, want) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return ER_ERR_NOMEM;
    }
    cap = want;
    return ER_OK;
}
void HostBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}

int set_error(er_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

int cuda_error(er_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return set_error(ctx, e == cudaErrorMemoryAllocation ? ER_ERR_NOMEM : ER_ERR_CUDA, m);
}

const FwRecord* find_fw(er_ctx* ctx, int fw_id) {
    auto it = ctx->fws.find(fw_id);
    return it == ctx->fws.end() ? nullptr : &it->second;
}

CutoffConsts make_cutoff_consts(double rc2, double /*box_diag*/, double r2min) {
    CutoffConsts c;
    const double rc = sqrt(rc2);
    const double m = 1e-3;
    c.rc = rc;
    c.rc2f = (float)rc2;
    c.rin2 = rc > 2 * m ? (float)((rc - m) * (rc - m)) : -1.0f;
    c.rout2 = (float)((rc + m) * (rc + m));
    c.rcm = rc + m;
    c.r2min = r2min;
    return c;
}

// ------------------------------------------------------------------ kernels
// Three CTAs per SM (24 warps): the FP32 variants fit 80 registers; the FP64
// variants (NEAR64, FP64) keep two.
template <int PREC>
constexpr int grid_min_blocks() {
    return (PREC == PREC_NEAR64 || PREC == PREC_FP64) ? 2 : 3;
}

template <int PREC, int P>
__global__ void __launch_bounds__(kThreads, grid_min_blocks<PREC>())
    grid_kernel(const __grid_constant__ GridTask task) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    EngineSmem& s = *reinterpret_cast<EngineSmem*>(smem_raw);
    GridPolicy<P> pol(&task, blockIdx.x);
    process_cta<GridPolicy<P>, PREC>(s, pol, task.fw, task.cc);
}

// One CTA per SM slot pulls (task, brick) items from the queue until it is
// empty; each task carries its own kernel variant (4 or 8 points per thread).
template <int PREC>
__global__ void __launch_bounds__(kThreads, grid_min_blocks<PREC>())
    grid_persistent_kernel(const GridTask* __restrict__ tasks, const WorkItem* __restrict__ items,
                           int n_items, int* head) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    EngineSmem& s = *reinterpret_cast<EngineSmem*>(smem_raw);
    for (;;) {
        if (threadIdx.x == 0) s.item = atomicAdd(head, 1);
        __syncthreads();
        const int it = s.item;
        __syncthreads();
        if (it >= n_items) break;
        const WorkItem wi = items[it];
        const GridTask* t = tasks + wi.task;
        if (t->tile_p == 8) {
            GridPolicy<8> pol(t, wi.brick);
            process_cta<GridPolicy<8>, PREC>(s, pol, t->fw, t->cc);
        } else {
            GridPolicy<4> pol(t, wi.brick);
            process_cta<GridPolicy<4>, PREC>(s, pol, t->fw, t->cc);
        }
    }
}

__global__ void f32_to_f64_kernel(const float* __restrict__ in, double* __restrict__ out,
                                  size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

template <int P>
static int configure_variant(er_ctx* ctx) {
    const int smem = (int)sizeof(EngineSmem);
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_kernel<PREC_COMP, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_kernel<PREC_FP32, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_kernel<PREC_COUNT, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_kernel<PREC_NEAR64, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_kernel<PREC_FP64, P>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return ER_OK;
}

static int configure_kernels(er_ctx* ctx) {
    int st = configure_variant<4>(ctx);
    if (st == ER_OK) st = configure_variant<8>(ctx);
    const int smem = (int)sizeof(EngineSmem);
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_persistent_kernel<PREC_COMP>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_persistent_kernel<PREC_FP32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return st;
}

int fill_grid_task(er_ctx* ctx, const FwRecord& fw, int nx, int ny, int nz, float* out,
                   GridTask& t, int tile_p) {
    if (tile_p != 4 && tile_p != 8)
        return set_error(ctx, ER_ERR_INVALID, "grid: kernel variant must have P = 4 or 8");
    if (nx < 2 || ny < 2 || nz < 2)
        return set_error(ctx, ER_ERR_INVALID, "grid: nx, ny, nz must be >= 2 (axes i/(N-1))");
    if ((double)nx * ny * nz > 4.0e9)
        return set_error(ctx, ER_ERR_LIMIT, "grid: more than 4e9 points");
    t.fw = fw.dev;
    t.cc = make_cutoff_consts(fw.rc2, 0.0, 1e-12 * 1e-12);  // min_r, src/computegridsheet.h:19
    t.nx = nx; t.ny = ny; t.nz = nz;
    t.tile_p = tile_p;
    t.nb[0] = (nx + 2 * tile_p - 1) / (2 * tile_p);
    t.nb[1] = (ny + 2 * kWJ - 1) / (2 * kWJ);
    t.nb[2] = (nz + 2 * kWK - 1) / (2 * kWK);
    t.out = out;
    t.out64 = nullptr;
    return ER_OK;
}

static int64_t task_bricks(const GridTask& t) { return (int64_t)t.nb[0] * t.nb[1] * t.nb[2]; }

int launch_grid_plain_on(er_ctx* ctx, const GridTask& t, int prec, cudaStream_t st) {
    const int64_t nbr = task_bricks(t);
    if (nbr > INT32_MAX) return set_error(ctx, ER_ERR_LIMIT, "grid: too many bricks");
    const size_t smem = sizeof(EngineSmem);
    const unsigned g = (unsigned)nbr;
    if (t.tile_p == 8) {
        if (prec == PREC_FP32) grid_kernel<PREC_FP32, 8><<<g, kThreads, smem, st>>>(t);
        else if (prec == PREC_COUNT) grid_kernel<PREC_COUNT, 8><<<g, kThreads, smem, st>>>(t);
        else if (prec == PREC_NEAR64) grid_kernel<PREC_NEAR64, 8><<<g, kThreads, smem, st>>>(t);
        else if (prec == PREC_FP64) grid_kernel<PREC_FP64, 8><<<g, kThreads, smem, st>>>(t);
        else grid_kernel<PREC_COMP, 8><<<g, kThreads, smem, st>>>(t);
    } else {
        if (prec == PREC_FP32) grid_kernel<PREC_FP32, 4><<<g, kThreads, smem, st>>>(t);
        else if (prec == PREC_COUNT) grid_kernel<PREC_COUNT, 4><<<g, kThreads, smem, st>>>(t);
        else if (prec == PREC_NEAR64) grid_kernel<PREC_NEAR64, 4><<<g, kThreads, smem, st>>>(t);
        else if (prec == PREC_FP64) grid_kernel<PREC_FP64, 4><<<g, kThreads, smem, st>>>(t);
        else grid_kernel<PREC_COMP, 4><<<g, kThreads, smem, st>>>(t);
    }
    ER_CUDA(ctx, cudaGetLastError());
    return ER_OK;
}

int launch_grid_plain(er_ctx* ctx, const GridTask& t, int prec) {
    return launch_grid_plain_on(ctx, t, prec, ctx->stream);
}

int launch_grid_persistent(er_ctx* ctx, const GridTask* d_tasks, const WorkItem* d_items,
                           int n_items, int* d_head, int prec) {
    const size_t smem = sizeof(EngineSmem);
    int per_sm = 0;
    ER_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                     &per_sm, grid_persistent_kernel<PREC_COMP>, kThreads, smem));
    per_sm = std::max(per_sm, 1);
    const int grid = std::min<int64_t>((int64_t)ctx->num_sms * per_sm, std::max(n_items, 1));
    ER_CUDA(ctx, cudaMemsetAsync(d_head, 0, sizeof(int), ctx->stream));
    cudaStream_t st = ctx->stream;
    if (prec == PREC_FP32)
        grid_persistent_kernel<PREC_FP32><<<grid, kThreads, smem, st>>>(d_tasks, d_items, n_items,
                                                                        d_head);
    else
        grid_persistent_kernel<PREC_COMP><<<grid, kThreads, smem, st>>>(d_tasks, d_items, n_items,
                                                                        d_head);
    ER_CUDA(ctx, cudaGetLastError());
    return ER_OK;
}

// ------------------------------------------------------------------ autotuner
// Picks the kernel variant (4 or 8 points per thread) for a class of jobs by
// timing both on the same sample of the job -- its first 16 x-layers, which
// are whole bricks for both variants -- and caches the faster one per class:
// (atoms per A^3 in half-octaves, smallest grid spacing in quarter-octaves,
// cutoff in quarter-Angstroms).
int tune_tile(er_ctx* ctx, const FwRecord& f, int nx, int ny, int nz, float* out, int* tile_p) {
    const double rho = (double)std::max(f.n_atoms, 1) / std::max(f.volume, 1e-9);
    double h = 1e30;
    const int dims[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) h = std::min(h, f.cell_len[d] / std::max(dims[d] - 1, 1));
    const std::tuple<int, int, int> key((int)lround(2.0 * log2(rho)), (int)lround(4.0 * log2(h)),
                                        (int)lround(4.0 * sqrt(f.rc2)));
    auto it = ctx->tune.find(key);
    if (it != ctx->tune.end()) {
        *tile_p = it->second;
        return ER_OK;
    }
    cudaEvent_t e0, e1;
    ER_CUDA(ctx, cudaEventCreate(&e0));
    ER_CUDA(ctx, cudaEventCreate(&e1));
    float best_ms = 0.f;
    int best = 4;
    // Both variants time the same first x-layers: a multiple of 16 large
    // enough for four waves of the bigger (P = 8) bricks on this GPU, so
    // neither variant is timed on an underfilled launch.
    const int nbyz = ((ny + 2 * kWJ - 1) / (2 * kWJ)) * ((nz + 2 * kWK - 1) / (2 * kWK));
    const int slots = 3 * ctx->num_sms;
    const int layers = 16 * std::max(1, (4 * slots + nbyz - 1) / nbyz);
    for (int P : {4, 8}) {
        GridTask t;
        int st = fill_grid_task(ctx, f, nx, ny, nz, out, t, P);
        if (st != ER_OK) return st;
        if (nx > layers) t.nb[0] = layers / (2 * P);
        float ms_min = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            ER_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
            st = launch_grid_plain(ctx, t, PREC_COMP);
            if (st != ER_OK) return st;
            ER_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
            ER_CUDA(ctx, cudaEventSynchronize(e1));
            float ms = 0.f;
            ER_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) ms_min = std::min(ms_min, ms);  // rep 0 warms up
        }
        if (P == 4 || ms_min < best_ms) {
            best_ms = ms_min;
            best = P;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->tune[key] = best;
    *tile_p = best;
    return ER_OK;
}

}  // namespace er

using namespace er;

// ------------------------------------------------------------------ C ABI
extern "C" {

int er_ctx_create(int device, er_ctx** out) {
    if (!out) return ER_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return ER_ERR_CUDA;
    }
    if (device < 0 || device >= n) return ER_ERR_INVALID;
    er_ctx* ctx = new er_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device) !=
            cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return ER_ERR_CUDA;
    }
    int st = configure_kernels(ctx);
    if (st != ER_OK) {
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return st;
    }
    *out = ctx;
    return ER_OK;
}

void er_ctx_destroy(er_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->fws) cudaFree(kv.second.block);
    ctx->fws.clear();
    DevBuf* bufs[] = {&ctx->grid_f32, &ctx->tasks,  &ctx->items,  &ctx->counter,
                      &ctx->p_grid,   &ctx->p_lab,  &ctx->p_seg,  &ctx->p_flags,
                      &ctx->p_misc,   &ctx->p_mask, &ctx->sheet_cache.grid};
    for (DevBuf* b : bufs) b->release();
    ctx->henry.release();
    ctx->pinned.release();
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* er_ctx_last_error(const er_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int er_ctx_synchronize(er_ctx* ctx) {
    if (!ctx) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return ER_OK;
}

int er_ctx_stream(er_ctx* ctx, void** stream) {
    if (!ctx || !stream) return ER_ERR_INVALID;
    *stream = (void*)ctx->stream;
    return ER_OK;
}

int er_framework_upload(er_ctx* ctx, const er_framework_desc* desc, int* fw_id) {
    if (!ctx || !desc || !fw_id) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    HostFramework hf;
    std::string err;
    int st = build_framework(*desc, ctx->cell_edge, hf, err);
    if (st != ER_OK) return set_error(ctx, st, err);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t n_img = hf.img_xyz.size();
    const size_t s_xyz = al(std::max<size_t>(n_img, 1) * sizeof(HostImage));
    const size_t s_par = al(std::max<size_t>(n_img, 1) * 2 * sizeof(float));
    const size_t s_id = al(std::max<size_t>(n_img, 1) * sizeof(uint32_t));
    const size_t s_cs = al(hf.cell_start.size() * sizeof(int));
    const size_t s_af = al(std::max<size_t>(hf.atom_frac.size(), 1) * sizeof(HostImage));
    const size_t s_lj = al(std::max<size_t>(hf.atom_lj64.size(), 2) * sizeof(double));
    const size_t total = s_xyz + s_par + s_id + s_cs + s_af + s_lj;
    FwRecord rec;
    if (cudaMalloc(&rec.block, total) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, ER_ERR_NOMEM, "framework upload: device allocation failed");
    }
    // one pinned host image of the whole block, one copy
    if (ctx->pinned.ensure(total) != ER_OK) {
        cudaFree(rec.block);
        return set_error(ctx, ER_ERR_NOMEM, "framework upload: pinned staging failed");
    }
    const size_t o_par = s_xyz, o_id = o_par + s_par, o_cs = o_id + s_id, o_af = o_cs + s_cs,
                 o_lj = o_af + s_af;
    char* h = (char*)ctx->pinned.ptr;
    memcpy(h, hf.img_xyz.data(), n_img * sizeof(HostImage));
    memcpy(h + o_par, hf.img_par.data(), n_img * 2 * sizeof(float));
    memcpy(h + o_id, hf.img_id.data(), n_img * sizeof(uint32_t));
    memcpy(h + o_cs, hf.cell_start.data(), hf.cell_start.size() * sizeof(int));
    memcpy(h + o_af, hf.atom_frac.data(), hf.atom_frac.size() * sizeof(HostImage));
    memcpy(h + o_lj, hf.atom_lj64.data(), hf.atom_lj64.size() * sizeof(double));
    cudaError_t e = cudaMemcpyAsync(rec.block, h, total, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(rec.block);
        return cuda_error(ctx, e, "framework upload: copy");
    }
    char* b = (char*)rec.block;
    FwDev& d = rec.dev;
    d.img_xyz = (const double4*)b;
    d.img_par = (const float2*)(b + o_par);
    d.img_id = (const uint32_t*)(b + o_id);
    d.cell_start = (const int*)(b + o_cs);
    d.atom_frac = (const double4*)(b + o_af);
    d.atom_lj64 = (const double2*)(b + o_lj);
    d.n_img = (int)n_img;
    d.n_atoms = hf.n_atoms;
    for (int k = 0; k < 3; ++k) {
        d.nc[k] = hf.nc[k];
        d.cell_lo[k] = hf.cell_lo[k];
        d.rep[k] = hf.rep[k];
    }
    d.h = hf.h;
    d.inv_h = 1.0 / hf.h;
    for (int k = 0; k < 9; ++k) d.t[k] = hf.t[k];
    for (int k = 0; k < 9; ++k) d.r[k] = hf.r[k];
    d.rc2 = hf.rc2;
    d.imgs_per_atom = hf.imgs_per_atom;
    rec.bytes = total;
    rec.rc2 = hf.rc2;
    for (int k = 0; k < 9; ++k) rec.t[k] = hf.t[k];
    for (int k = 0; k < 3; ++k)
        rec.cell_len[k] = sqrt(hf.t[k] * hf.t[k] + hf.t[3 + k] * hf.t[3 + k] +
                               hf.t[6 + k] * hf.t[6 + k]);
    rec.volume = fabs(hf.t[0] * (hf.t[4] * hf.t[8] - hf.t[5] * hf.t[7]) -
                      hf.t[1] * (hf.t[3] * hf.t[8] - hf.t[5] * hf.t[6]) +
                      hf.t[2] * (hf.t[3] * hf.t[7] - hf.t[4] * hf.t[6]));
    rec.n_atoms = hf.n_atoms;
    const int id = ctx->next_fw++;
    ctx->fws[id] = rec;
    *fw_id = id;
    return ER_OK;
}

int er_framework_release(er_ctx* ctx, int fw_id) {
    if (!ctx) return ER_ERR_INVALID;
    auto it = ctx->fws.find(fw_id);
    if (it == ctx->fws.end()) return set_error(ctx, ER_ERR_NOT_FOUND, "unknown framework id");
    cudaStreamSynchronize(ctx->stream);
    cudaFree(it->second.block);
    ctx->fws.erase(it);
    if (ctx->sheet_cache.fw == fw_id) ctx->sheet_cache.fw = 0;
    return ER_OK;
}

int er_framework_bytes(er_ctx* ctx, int fw_id, size_t* bytes) {
    if (!ctx || !bytes) return ER_ERR_INVALID;
    const FwRecord* f = find_fw(ctx, fw_id);
    if (!f) return set_error(ctx, ER_ERR_NOT_FOUND, "unknown framework id");
    *bytes = f->bytes;
    return ER_OK;
}

int er_grid(er_ctx* ctx, int fw_id, int nx, int ny, int nz, int flags, void* out) {
    if (!ctx || !out) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    const FwRecord* f = find_fw(ctx, fw_id);
    if (!f) return set_error(ctx, ER_ERR_NOT_FOUND, "grid: unknown framework id");
    const int tile_p = (flags & ER_TILE_P8) ? 8 : 4;
    const int prec = (flags & ER_COUNT_PAIRS)   ? PREC_COUNT
                     : (flags & ER_PREC_FP32)   ? PREC_FP32
                     : (flags & ER_PREC_NEAR64) ? PREC_NEAR64
                                                : PREC_COMP;
    const size_t npts = (size_t)nx * ny * nz;
    const bool dev_out = (flags & ER_OUT_DEVICE) != 0;
    const bool f64 = (flags & ER_OUT_F64) != 0;
    if (flags & ER_PREC_FP64) {
        // FP64 pair terms and sums, written as FP64
        if (!f64)
            return set_error(ctx, ER_ERR_INVALID, "grid: ER_PREC_FP64 needs ER_OUT_F64");
        if (flags & (ER_COUNT_PAIRS | ER_PREC_FP32 | ER_PREC_NEAR64))
            return set_error(ctx, ER_ERR_INVALID, "grid: conflicting precision flags");
        double* d64 = (double*)out;
        if (!dev_out) {
            if (ctx->grid_f32.ensure(npts * sizeof(double)) != ER_OK)
                return set_error(ctx, ER_ERR_NOMEM, "grid: staging allocation failed");
            d64 = (double*)ctx->grid_f32.ptr;
        }
        GridTask t;
        int st = fill_grid_task(ctx, *f, nx, ny, nz, nullptr, t, tile_p);
        if (st != ER_OK) return st;
        t.out64 = d64;
        st = launch_grid_plain(ctx, t, PREC_FP64);
        if (st != ER_OK) return st;
        if (!dev_out) {
            ER_CUDA(ctx, cudaMemcpyAsync(out, d64, npts * sizeof(double), cudaMemcpyDeviceToHost,
                                         ctx->stream));
            ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        return ER_OK;
    }
    float* dst = nullptr;
    if (dev_out && !f64) {
        dst = (float*)out;
    } else {
        if (ctx->grid_f32.ensure(npts * sizeof(float)) != ER_OK)
            return set_error(ctx, ER_ERR_NOMEM, "grid: staging allocation failed");
        dst = (float*)ctx->grid_f32.ptr;
    }
    GridTask t;
    int st = fill_grid_task(ctx, *f, nx, ny, nz, dst, t, tile_p);
    if (st != ER_OK) return st;
    st = launch_grid_plain(ctx, t, prec);
    if (st != ER_OK) return st;
    if (dev_out && f64) {
        f32_to_f64_kernel<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(dst, (double*)out, npts);
        ER_CUDA(ctx, cudaGetLastError());
    } else if (!dev_out) {
        if (!f64) {
            ER_CUDA(ctx, cudaMemcpyAsync(out, dst, npts * sizeof(float), cudaMemcpyDeviceToHost,
                                         ctx->stream));
            ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        } else {
            // D2H as float (half the bytes), widen on the host
            float* tmp = (float*)out;  // the first half of the caller's double buffer
            ER_CUDA(ctx, cudaMemcpyAsync(tmp, dst, npts * sizeof(float), cudaMemcpyDeviceToHost,
                                         ctx->stream));
            ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            double* o = (double*)out;
            for (size_t i = npts; i-- > 0;) o[i] = (double)tmp[i];
        }
    }
    return ER_OK;
}

int er_grid_sheet(er_ctx* ctx, int fw_id, int nx, int ny, int nz, int x_index,
                  double* out_sheet) {
    if (!ctx || !out_sheet) return ER_ERR_INVALID;
    if (x_index < 0 || x_index >= nx) return set_error(ctx, ER_ERR_INVALID, "sheet: x_index");
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    auto& c = ctx->sheet_cache;
    const size_t npts = (size_t)nx * ny * nz;
    if (!(c.fw == fw_id && c.nx == nx && c.ny == ny && c.nz == nz)) {
        c.fw = 0;
        if (c.grid.ensure(npts * sizeof(float)) != ER_OK)
            return set_error(ctx, ER_ERR_NOMEM, "sheet: grid cache allocation failed");
        int st = er_grid(ctx, fw_id, nx, ny, nz, ER_OUT_DEVICE | ER_OUT_F32, c.grid.ptr);
        if (st != ER_OK) return st;
        c.fw = fw_id; c.nx = nx; c.ny = ny; c.nz = nz;
    }
    const size_t ns = (size_t)ny * nz;
    if (ctx->pinned.ensure(ns * sizeof(float)) != ER_OK)
        return set_error(ctx, ER_ERR_NOMEM, "sheet: pinned staging failed");
    ER_CUDA(ctx, cudaMemcpyAsync(ctx->pinned.ptr, (float*)c.grid.ptr + (size_t)x_index * ns,
                                 ns * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const float* src = (const float*)ctx->pinned.ptr;
    for (size_t i = 0; i < ns; ++i) out_sheet[i] = (double)src[i];
    return ER_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batches
struct er_batch_plan {
    er_ctx* ctx = nullptr;
    int mode = ER_BATCH_PERSISTENT;
    int n_jobs = 0;
    std::vector<GridTask> tasks;
    GridTask* d_tasks = nullptr;
    WorkItem* d_items = nullptr;
    int n_items = 0;
    int* d_head = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
};

namespace er {

// Longest-first order of (task, brick) items: bricks of denser frameworks and
// bigger grids first, so the persistent queue drains with a short tail.
static void build_items(const std::vector<GridTask>& tasks, const std::vector<double>& cost,
                        std::vector<WorkItem>& items) {
    std::vector<int> order(tasks.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    items.clear();
    for (int ti : order) {
        const int64_t nb = task_bricks(tasks[ti]);
        for (int64_t b = 0; b < nb; ++b) items.push_back(WorkItem{ti, (int)b});
    }
}

static int plan_enqueue(er_batch_plan* p) {
    er_ctx* ctx = p->ctx;
    if (p->mode == ER_BATCH_PLAIN) {
        for (int i = 0; i < p->n_jobs; ++i) {
            int st = launch_grid_plain(ctx, p->tasks[i], PREC_COMP);
            if (st != ER_OK) return st;
        }
        return ER_OK;
    }
    return launch_grid_persistent(ctx, p->d_tasks, p->d_items, p->n_items, p->d_head, PREC_COMP);
}

}  // namespace er

extern "C" {

int er_batch_plan_create(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode,
                         er_batch_plan** out) {
    if (!ctx || !out || (n_jobs > 0 && !jobs) || n_jobs < 0) return ER_ERR_INVALID;
    const bool autotune = (mode & ER_BATCH_AUTOTUNE) != 0;
    mode &= ~ER_BATCH_AUTOTUNE;
    if (mode != ER_BATCH_PERSISTENT && mode != ER_BATCH_PLAIN) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    *out = nullptr;
    er_batch_plan* p = new er_batch_plan();
    p->ctx = ctx;
    p->mode = mode;
    p->n_jobs = n_jobs;
    std::vector<double> cost;
    for (int i = 0; i < n_jobs; ++i) {
        const FwRecord* f = find_fw(ctx, jobs[i].fw_id);
        if (!f || !jobs[i].out_device) {
            delete p;
            return set_error(ctx, f ? ER_ERR_INVALID : ER_ERR_NOT_FOUND,
                             "batch: unknown framework id or NULL output");
        }
        int tile_p = 4;
        int st = ER_OK;
        if (autotune && jobs[i].nx >= 2 && jobs[i].ny >= 2 && jobs[i].nz >= 2)
            st = tune_tile(ctx, *f, jobs[i].nx, jobs[i].ny, jobs[i].nz, jobs[i].out_device,
                           &tile_p);
        GridTask t;
        if (st == ER_OK)
            st = fill_grid_task(ctx, *f, jobs[i].nx, jobs[i].ny, jobs[i].nz, jobs[i].out_device, t,
                                tile_p);
        if (st != ER_OK) {
            delete p;
            return st;
        }
        p->tasks.push_back(t);
        // per-brick cost ~ atom density * cutoff volume
        cost.push_back((double)f->dev.n_img / std::max(1.0, f->volume));
    }
    std::vector<WorkItem> items;
    build_items(p->tasks, cost, items);
    p->n_items = (int)items.size();
    auto fail = [&](int st, const char* m) {
        er_batch_plan_destroy(p);
        return set_error(ctx, st, m);
    };
    if (cudaMalloc(&p->d_tasks, std::max<size_t>(1, p->tasks.size()) * sizeof(GridTask)) !=
            cudaSuccess ||
        cudaMalloc(&p->d_items, std::max<size_t>(1, items.size()) * sizeof(WorkItem)) !=
            cudaSuccess ||
        cudaMalloc(&p->d_head, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return fail(ER_ERR_NOMEM, "batch: device allocation failed");
    }
    if (!p->tasks.empty() &&
        cudaMemcpy(p->d_tasks, p->tasks.data(), p->tasks.size() * sizeof(GridTask),
                   cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(ER_ERR_CUDA, "batch: task upload failed");
    if (!items.empty() && cudaMemcpy(p->d_items, items.data(), items.size() * sizeof(WorkItem),
                                     cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(ER_ERR_CUDA, "batch: queue upload failed");
    // capture the launch sequence once as a CUDA graph
    cudaStream_t cs = ctx->stream;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(ER_ERR_CUDA, "batch: stream capture failed");
    int st = plan_enqueue(p);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    if (st != ER_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return fail(ER_ERR_CUDA, "batch: graph capture failed");
    }
    p->graph = g;
    if (cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) {
        cudaGetLastError();
        return fail(ER_ERR_CUDA, "batch: graph instantiation failed");
    }
    size_t n_nodes = 0;
    cudaGraphGetNodes(g, nullptr, &n_nodes);
    std::vector<cudaGraphNode_t> nodes(n_nodes);
    if (n_nodes) cudaGraphGetNodes(g, nodes.data(), &n_nodes);
    int kn = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType ty;
        cudaGraphNodeGetType(nd, &ty);
        if (ty == cudaGraphNodeTypeKernel) ++kn;
    }
    p->launches = kn;
    *out = p;
    return ER_OK;
}

int er_batch_plan_run(er_batch_plan* p) {
    if (!p) return ER_ERR_INVALID;
    ER_CUDA(p->ctx, cudaGraphLaunch(p->exec, p->ctx->stream));
    return ER_OK;
}

int er_batch_plan_launches(const er_batch_plan* p, int* n) {
    if (!p || !n) return ER_ERR_INVALID;
    *n = p->launches;
    return ER_OK;
}

int er_batch_plan_tile(const er_batch_plan* p, int job, int* tile_p) {
    if (!p || !tile_p || job < 0 || job >= p->n_jobs) return ER_ERR_INVALID;
    *tile_p = p->tasks[job].tile_p;
    return ER_OK;
}

void er_batch_plan_destroy(er_batch_plan* p) {
    if (!p) return;
    if (p->ctx) cudaStreamSynchronize(p->ctx->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->d_tasks) cudaFree(p->d_tasks);
    if (p->d_items) cudaFree(p->d_items);
    if (p->d_head) cudaFree(p->d_head);
    delete p;
}

int er_grid_batch(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode) {
    if (!ctx || n_jobs < 0 || (n_jobs > 0 && !jobs)) return ER_ERR_INVALID;
    if (mode & ER_BATCH_HOST_OUT) {
        // stage every grid in one device buffer, run, copy each back
        std::vector<er_grid_job> dj(jobs, jobs + n_jobs);
        std::vector<size_t> off(n_jobs + 1, 0);
        for (int i = 0; i < n_jobs; ++i) {
            if (jobs[i].nx < 2 || jobs[i].ny < 2 || jobs[i].nz < 2 || !jobs[i].out_device)
                return set_error(ctx, ER_ERR_INVALID, "batch: bad job dims or NULL output");
            off[i + 1] = off[i] + (size_t)jobs[i].nx * jobs[i].ny * jobs[i].nz;
        }
        ER_CUDA(ctx, cudaSetDevice(ctx->device));
        if (ctx->grid_f32.ensure(std::max<size_t>(off[n_jobs], 1) * sizeof(float)) != ER_OK)
            return set_error(ctx, ER_ERR_NOMEM, "batch: device staging allocation failed");
        float* base = (float*)ctx->grid_f32.ptr;
        for (int i = 0; i < n_jobs; ++i) dj[i].out_device = base + off[i];
        int st = er_grid_batch(ctx, dj.data(), n_jobs, mode & ~ER_BATCH_HOST_OUT);
        if (st != ER_OK) return st;
        for (int i = 0; i < n_jobs; ++i)
            ER_CUDA(ctx, cudaMemcpyAsync(jobs[i].out_device, base + off[i],
                                         (off[i + 1] - off[i]) * sizeof(float),
                                         cudaMemcpyDeviceToHost, ctx->stream));
        ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return ER_OK;
    }
    er_batch_plan* p = nullptr;
    int st = er_batch_plan_create(ctx, jobs, n_jobs, mode, &p);
    if (st != ER_OK) return st;
    st = er_batch_plan_run(p);
    if (st == ER_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        st = cuda_error(ctx, cudaGetLastError(), "batch: run");
    er_batch_plan_destroy(p);
    return st;
}

}  // extern "C"

// ------------------------------------------------------------------ diagnostics
namespace er {

// 8 independent FFMA chains per thread; the final values are stored only when
// a data-dependent test that never holds is true, so the chains stay live.
__global__ void __launch_bounds__(256) fp32_rate_kernel(int iters, float seed, float* sink) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = __fmaf_rn(a0, m, c); a1 = __fmaf_rn(a1, m, c);
            a2 = __fmaf_rn(a2, m, c); a3 = __fmaf_rn(a3, m, c);
            a4 = __fmaf_rn(a4, m, c); a5 = __fmaf_rn(a5, m, c);
            a6 = __fmaf_rn(a6, m, c); a7 = __fmaf_rn(a7, m, c);
        }
    }
    const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == -1.2345f) sink[blockIdx.x] = r;
}

}  // namespace er

extern "C" int er_probe_fp32_rate(er_ctx* ctx, double seconds, double* instr_per_s) {
    if (!ctx || !instr_per_s || !(seconds > 0)) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->counter.ensure(4096 * sizeof(float)) != ER_OK)
        return set_error(ctx, ER_ERR_NOMEM, "probe: allocation failed");
    const int blocks = ctx->num_sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    ER_CUDA(ctx, cudaEventCreate(&e0));
    ER_CUDA(ctx, cudaEventCreate(&e1));
    int iters = 256;
    double best = 0.0;
    for (int round = 0; round < 12; ++round) {
        ER_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
        fp32_rate_kernel<<<blocks, threads, 0, ctx->stream>>>(iters, 1.0f, (float*)ctx->counter.ptr);
        ER_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
        ER_CUDA(ctx, cudaEventSynchronize(e1));
        float ms = 0.f;
        ER_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
        const double inst = (double)blocks * threads * iters * 16.0 * 8.0;
        if (ms > 0) best = std::max(best, inst / (ms * 1e-3));
        if (ms * 1e-3 < seconds / 4 && iters < (1 << 26)) iters *= 2;
        else if (round >= 6) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *instr_per_s = best;
    return ER_OK;
}
