// er_api.cu -- context, framework upload and the grid entry points of the C ABI.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "er_ctx.h"
#include "er_nvtx.h"
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
int DevBuf::ensure_on(size_t bytes, cudaMemPool_t pool, cudaStream_t st) {
    if (bytes <= cap && ptr) return ER_OK;
    if (ptr) {
        if (owner) cudaFreeAsync(ptr, owner);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    cap = 0;
    owner = nullptr;
    size_t want = std::max<size_t>(bytes, 256);
    if (cudaMallocFromPoolAsync(&ptr, want, pool, st) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return ER_ERR_NOMEM;
    }
    cap = want;
    owner = st;
    return ER_OK;
}
void DevBuf::release() {
    if (ptr) {
        if (owner) cudaFreeAsync(ptr, owner);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    cap = 0;
    owner = nullptr;
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
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->err_mu);
        ctx->last_error = msg;
    }
    return status;
}

int take_fault(er_ctx* ctx) {
    if (!ctx->fault_host || !*(volatile int*)ctx->fault_host) return ER_OK;
    *(volatile int*)ctx->fault_host = 0;
    return set_error(ctx, ER_ERR_CUDA,
                     "engine: a bounded wait for staged atom images gave up; the grid points "
                     "or insertions of the affected blocks were not written");
}

int cuda_error(er_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return set_error(ctx, e == cudaErrorMemoryAllocation ? ER_ERR_NOMEM : ER_ERR_CUDA, m);
}

int pool_alloc(er_ctx* ctx, void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), ctx->pool, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaStreamSynchronize(ctx->stream);
        cudaMemPoolTrimTo(ctx->pool, 0);
        e = cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), ctx->pool, ctx->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return ER_ERR_NOMEM;
        }
    }
    return ER_OK;
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
// Three CTAs per SM (24 warps) at 80 registers. NEAR64 spills some of its
// FP64 near-pair state at that limit and is still faster than at two CTAs
// (128 registers): 385.5 against 399.2 ms on the 256-framework batch. FP64
// (all pairs in FP64, a reference mode) keeps two.
template <int PREC>
constexpr int grid_min_blocks() {
    return PREC == PREC_FP64 ? 2 : 3;
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
// With task_left given, the CTA that finishes a task's last brick raises the
// task's flag in host-mapped memory (done_host), so the host can copy that
// grid out while the kernel runs on.
// Queue item q is brick q - start[k] of task k, start[k] <= q < start[k + 1];
// tasks are stored longest first.
template <int PREC>
__global__ void __launch_bounds__(kThreads, grid_min_blocks<PREC>())
    grid_persistent_kernel(const GridTask* __restrict__ tasks, const int* __restrict__ start,
                           int n_tasks, int n_items, int* head, int* task_left,
                           volatile int* done_host) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    EngineSmem& s = *reinterpret_cast<EngineSmem*>(smem_raw);
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(head, 1);
            int k = 0;
            if (it < n_items) {
                int hi = n_tasks - 1;
                while (k < hi) {
                    const int mid = (k + hi + 1) >> 1;
                    if (start[mid] <= it) k = mid; else hi = mid - 1;
                }
            }
            s.item = it;
            s.task = k;
        }
        __syncthreads();
        const int it = s.item;
        const WorkItem wi{s.task, it < n_items ? it - start[s.task] : 0};
        __syncthreads();
        if (it >= n_items) break;
        const GridTask* t = tasks + wi.task;
        if (t->tile_p == 8) {
            GridPolicy<8> pol(t, wi.brick);
            process_cta<GridPolicy<8>, PREC>(s, pol, t->fw, t->cc);
        } else {
            GridPolicy<4> pol(t, wi.brick);
            process_cta<GridPolicy<4>, PREC>(s, pol, t->fw, t->cc);
        }
        if (task_left) {
            __threadfence();  // this thread's grid stores, device-wide
            __syncthreads();
            if (threadIdx.x == 0 && atomicSub(&task_left[wi.task], 1) == 1) {
                __threadfence_system();
                done_host[wi.task] = 1;
            }
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
    ER_CUDA(ctx, cudaFuncSetAttribute(grid_persistent_kernel<PREC_NEAR64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return st;
}

int check_grid_dims(er_ctx* ctx, int nx, int ny, int nz, const char* who) {
    if (nx < 2 || ny < 2 || nz < 2)
        return set_error(ctx, ER_ERR_INVALID,
                         std::string(who) + ": nx, ny, nz must be >= 2 (axes i/(N-1))");
    if ((double)nx * ny * nz > 4.0e9)
        return set_error(ctx, ER_ERR_LIMIT, std::string(who) + ": more than 4e9 points");
    return ER_OK;
}

int fill_grid_task(er_ctx* ctx, const FwRecord& fw, int nx, int ny, int nz, float* out,
                   GridTask& t, int tile_p) {
    if (tile_p != 4 && tile_p != 8)
        return set_error(ctx, ER_ERR_INVALID, "grid: kernel variant must have P = 4 or 8");
    if (int st = check_grid_dims(ctx, nx, ny, nz, "grid")) return st;
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

int launch_grid_persistent(er_ctx* ctx, const GridTask* d_tasks, const int* d_start, int n_tasks,
                           int n_items, int* d_head, int prec, int* task_left = nullptr,
                           int* done_dev = nullptr) {
    const size_t smem = sizeof(EngineSmem);
    int per_sm = 0;
    ER_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                     &per_sm,
                     prec == PREC_NEAR64 ? grid_persistent_kernel<PREC_NEAR64>
                                         : grid_persistent_kernel<PREC_COMP>,
                     kThreads, smem));
    per_sm = std::max(per_sm, 1);
    const int grid = std::min<int64_t>((int64_t)ctx->num_sms * per_sm, std::max(n_items, 1));
    ER_CUDA(ctx, cudaMemsetAsync(d_head, 0, sizeof(int), ctx->stream));
    cudaStream_t st = ctx->stream;
    if (prec == PREC_FP32)
        grid_persistent_kernel<PREC_FP32><<<grid, kThreads, smem, st>>>(
            d_tasks, d_start, n_tasks, n_items, d_head, task_left, done_dev);
    else if (prec == PREC_NEAR64)
        grid_persistent_kernel<PREC_NEAR64><<<grid, kThreads, smem, st>>>(
            d_tasks, d_start, n_tasks, n_items, d_head, task_left, done_dev);
    else
        grid_persistent_kernel<PREC_COMP><<<grid, kThreads, smem, st>>>(
            d_tasks, d_start, n_tasks, n_items, d_head, task_left, done_dev);
    ER_CUDA(ctx, cudaGetLastError());
    return ER_OK;
}

// ------------------------------------------------------------------ autotuner
// Picks the kernel variant (4 or 8 points per thread) for a class of jobs by
// timing both, in the precision mode the jobs run in, on the same sample of
// the job -- its first 16 x-layers, which are whole bricks for both variants
// -- and caches the faster one per class: (atoms per A^3 in half-octaves,
// smallest grid spacing in quarter-octaves, cutoff in quarter-Angstroms,
// precision mode).
int tune_tile(er_ctx* ctx, const FwRecord& f, int nx, int ny, int nz, float* out, int prec,
              int* tile_p) {
    const double rho = (double)std::max(f.n_atoms, 1) / std::max(f.volume, 1e-9);
    double h = 1e30;
    const int dims[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d) h = std::min(h, f.cell_len[d] / std::max(dims[d] - 1, 1));
    const std::tuple<int, int, int, int> key((int)lround(2.0 * log2(rho)),
                                             (int)lround(4.0 * log2(h)),
                                             (int)lround(4.0 * sqrt(f.rc2)), prec);
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
            st = launch_grid_plain(ctx, t, prec);
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
    if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return ER_ERR_CUDA;
    }
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool
        // no reuse that would make one stream wait for another's pending free
        int no_dep = 0;
        if (cudaMemPoolCreate(&ctx->pool, &props) != cudaSuccess ||
            cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep) !=
                cudaSuccess ||
            cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolReuseAllowInternalDependencies,
                                    &no_dep) != cudaSuccess) {
            cudaGetLastError();
            if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
            cudaStreamDestroy(ctx->copy_stream);
            cudaStreamDestroy(ctx->stream);
            delete ctx;
            return ER_ERR_CUDA;
        }
    }
    int st = configure_kernels(ctx);
    if (st == ER_OK) {
        if (cudaHostAlloc((void**)&ctx->fault_host, sizeof(int), cudaHostAllocMapped) !=
                cudaSuccess ||
            cudaHostGetDevicePointer((void**)&ctx->fault_dev, ctx->fault_host, 0) !=
                cudaSuccess) {
            cudaGetLastError();
            st = ER_ERR_CUDA;
        } else {
            *ctx->fault_host = 0;
        }
    }
    if (st != ER_OK) {
        if (ctx->fault_host) cudaFreeHost(ctx->fault_host);
        cudaMemPoolDestroy(ctx->pool);
        cudaStreamDestroy(ctx->copy_stream);
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
    cudaStreamSynchronize(ctx->copy_stream);
    for (auto& kv : ctx->fws) cudaFreeAsync(kv.second.block, ctx->stream);
    ctx->fws.clear();
    DevBuf* bufs[] = {&ctx->grid_f32, &ctx->counter, &ctx->sheet_cache.grid, &ctx->interp};
    for (DevBuf* b : bufs) b->release();
    ctx->pocket.release();
    for (HenryPipe* p : ctx->pipes) {
        cudaStreamSynchronize(p->stream);
        p->hs.release();
        p->ps.release();
        p->grid.release();
        p->mask.release();
        cudaStreamSynchronize(p->stream);
        if (p->out) cudaFreeHost(p->out);
        cudaStreamDestroy(p->stream);
        delete p;
    }
    ctx->pipes.clear();
    ctx->henry.release();
    for (cudaEvent_t& e : ctx->henry.ev)
        if (e) cudaEventDestroy(e);
    ctx->pinned.release();
    ctx->plan_pinned.release();
    ctx->task_left.release();
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolDestroy(ctx->pool);
    if (ctx->done_host) cudaFreeHost(ctx->done_host);
    if (ctx->fault_host) cudaFreeHost(ctx->fault_host);
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* er_ctx_last_error(const er_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int er_ctx_synchronize(er_ctx* ctx) {
    if (!ctx) return ER_ERR_INVALID;
    ER_SYNC(ctx, ctx->stream);
    return ER_OK;
}

int er_ctx_stream(er_ctx* ctx, void** stream) {
    if (!ctx || !stream) return ER_ERR_INVALID;
    *stream = (void*)ctx->stream;
    return ER_OK;
}

}  // extern "C"

namespace er {

FwLayout fw_layout(size_t n_img, size_t n_cs, size_t n_atoms) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    FwLayout L;
    const size_t s_xyz = al(std::max<size_t>(n_img, 1) * sizeof(HostImage));
    const size_t s_par = al(std::max<size_t>(n_img, 1) * 2 * sizeof(float));
    const size_t s_id = al(std::max<size_t>(n_img, 1) * sizeof(uint32_t));
    const size_t s_cs = al(n_cs * sizeof(int));
    const size_t s_af = al(std::max<size_t>(n_atoms, 1) * sizeof(HostImage));
    const size_t s_lj = al(std::max<size_t>(2 * n_atoms, 2) * sizeof(double));
    const size_t s_ilj = al(std::max<size_t>(n_img, 1) * 2 * sizeof(double));
    L.o_par = s_xyz;
    L.o_id = L.o_par + s_par;
    L.o_cs = L.o_id + s_id;
    L.o_af = L.o_cs + s_cs;
    L.o_lj = L.o_af + s_af;
    L.o_ilj = L.o_lj + s_lj;
    L.total = L.o_ilj + s_ilj;
    return L;
}

// Writes the host image of the device block at h.
static void fw_stage(const HostFramework& hf, const FwLayout& L, char* h) {
    const size_t n_img = hf.img_xyz.size();
    memcpy(h, hf.img_xyz.data(), n_img * sizeof(HostImage));
    memcpy(h + L.o_par, hf.img_par.data(), n_img * 2 * sizeof(float));
    memcpy(h + L.o_id, hf.img_id.data(), n_img * sizeof(uint32_t));
    memcpy(h + L.o_cs, hf.cell_start.data(), hf.cell_start.size() * sizeof(int));
    memcpy(h + L.o_af, hf.atom_frac.data(), hf.atom_frac.size() * sizeof(HostImage));
    memcpy(h + L.o_lj, hf.atom_lj64.data(), hf.atom_lj64.size() * sizeof(double));
    memcpy(h + L.o_ilj, hf.img_lj64.data(), n_img * 2 * sizeof(double));
}

// Fills the handle record of a framework whose block is (being) written at `block`.
void fw_record(const HostFramework& hf, size_t n_img, const FwLayout& L, void* block,
               FwRecord& rec) {
    rec.block = block;
    char* b = (char*)block;
    FwDev& d = rec.dev;
    d.img_xyz = (const double4*)b;
    d.img_par = (const float2*)(b + L.o_par);
    d.img_id = (const uint32_t*)(b + L.o_id);
    d.cell_start = (const int*)(b + L.o_cs);
    d.atom_frac = (const double4*)(b + L.o_af);
    d.atom_lj64 = (const double2*)(b + L.o_lj);
    d.img_lj64 = (const double2*)(b + L.o_ilj);
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
    d.fault = nullptr;
    rec.bytes = L.total;
    rec.rc2 = hf.rc2;
    for (int k = 0; k < 9; ++k) rec.t[k] = hf.t[k];
    for (int k = 0; k < 3; ++k)
        rec.cell_len[k] = sqrt(hf.t[k] * hf.t[k] + hf.t[3 + k] * hf.t[3 + k] +
                               hf.t[6 + k] * hf.t[6 + k]);
    rec.volume = fabs(hf.t[0] * (hf.t[4] * hf.t[8] - hf.t[5] * hf.t[7]) -
                      hf.t[1] * (hf.t[3] * hf.t[8] - hf.t[5] * hf.t[6]) +
                      hf.t[2] * (hf.t[3] * hf.t[7] - hf.t[4] * hf.t[6]));
    rec.n_atoms = hf.n_atoms;
}

}  // namespace er

extern "C" {

int er_framework_upload(er_ctx* ctx, const er_framework_desc* desc, int* fw_id) {
    er::NvtxRange nvtx("er_framework_upload");
    if (!ctx || !desc || !fw_id) return ER_ERR_INVALID;
    return host_upload_many(ctx, desc, 1, fw_id);
}

int er_framework_upload_many(er_ctx* ctx, const er_framework_desc* descs, int n, int* fw_ids) {
    er::NvtxRange nvtx("er_framework_upload_many");
    if (!ctx || n < 0 || (n > 0 && (!descs || !fw_ids))) return ER_ERR_INVALID;
    if (n == 0) return ER_OK;
    return device_upload_many(ctx, descs, n, fw_ids);
}

}  // extern "C"

namespace er {

// Uploads with the image cell lists built on the host threads (one framework
// per thread), staged into pinned memory and copied.
int host_upload_many(er_ctx* ctx, const er_framework_desc* descs, int n, int* fw_ids) {
    if (n == 0) return ER_OK;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    // 1. image cell lists, built on the host threads
    std::vector<HostFramework> hfs(n);
    std::vector<std::string> errs(n);
    std::vector<int> sts(n, ER_OK);
    const double h = ctx->cell_edge;
    parallel_for(n, [&](int i) { sts[i] = build_framework(descs[i], h, hfs[i], errs[i]); });
    for (int i = 0; i < n; ++i)
        if (sts[i] != ER_OK)
            return set_error(ctx, sts[i],
                             n > 1 ? "framework " + std::to_string(i) + ": " + errs[i] : errs[i]);
    // 2. device blocks and one pinned host image of all of them
    std::vector<FwLayout> lay(n);
    std::vector<size_t> at(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        lay[i] = fw_layout(hfs[i].img_xyz.size(), hfs[i].cell_start.size(), hfs[i].atom_frac.size());
        at[i + 1] = at[i] + lay[i].total;
    }
    std::vector<void*> blocks(n, nullptr);
    auto free_blocks = [&]() {
        cudaStreamSynchronize(ctx->stream);
        for (void* b : blocks)
            if (b) cudaFreeAsync(b, ctx->stream);
    };
    for (int i = 0; i < n; ++i)
        if (pool_alloc(ctx, &blocks[i], lay[i].total) != ER_OK) {
            free_blocks();
            return set_error(ctx, ER_ERR_NOMEM, "framework upload: device allocation failed");
        }
    if (ctx->pinned.ensure(at[n]) != ER_OK) {
        free_blocks();
        return set_error(ctx, ER_ERR_NOMEM, "framework upload: pinned staging failed");
    }
    char* h0 = (char*)ctx->pinned.ptr;
    parallel_for(n, [&](int i) { fw_stage(hfs[i], lay[i], h0 + at[i]); });
    // 3. one copy per framework, one wait
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < n && e == cudaSuccess; ++i)
        e = cudaMemcpyAsync(blocks[i], h0 + at[i], lay[i].total, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(ctx->stream);
        free_blocks();
        return cuda_error(ctx, e, "framework upload: copy");
    }
    for (int i = 0; i < n; ++i) {
        FwRecord rec;
        fw_record(hfs[i], hfs[i].img_xyz.size(), lay[i], blocks[i], rec);
        rec.dev.fault = ctx->fault_dev;
        const int id = ctx->next_fw++;
        ctx->fws[id] = rec;
        fw_ids[i] = id;
    }
    return ER_OK;
}

}  // namespace er

extern "C" {

int er_framework_release(er_ctx* ctx, int fw_id) {
    if (!ctx) return ER_ERR_INVALID;
    auto it = ctx->fws.find(fw_id);
    if (it == ctx->fws.end()) return set_error(ctx, ER_ERR_NOT_FOUND, "unknown framework id");
    // no work of this process may still read the block (as with cudaFree)
    cudaDeviceSynchronize();
    cudaFreeAsync(it->second.block, ctx->stream);
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
    er::NvtxRange nvtx("er_grid");
    if (!ctx || !out) return ER_ERR_INVALID;
    if (int st = check_grid_dims(ctx, nx, ny, nz, "grid")) return st;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    const FwRecord* f = find_fw(ctx, fw_id);
    if (!f) return set_error(ctx, ER_ERR_NOT_FOUND, "grid: unknown framework id");
    const int tile_p = (flags & ER_TILE_P8) ? 8 : 4;
    const int prec = (flags & ER_COUNT_PAIRS) ? PREC_COUNT
                     : (flags & ER_PREC_FP32) ? PREC_FP32
                     : (flags & ER_PREC_COMP) ? PREC_COMP
                                              : PREC_NEAR64;
    const size_t npts = (size_t)nx * ny * nz;
    const bool dev_out = (flags & ER_OUT_DEVICE) != 0;
    const bool f64 = (flags & ER_OUT_F64) != 0;
    if (flags & ER_PREC_FP64) {
        // FP64 pair terms and sums, written as FP64
        if (!f64)
            return set_error(ctx, ER_ERR_INVALID, "grid: ER_PREC_FP64 needs ER_OUT_F64");
        if (flags & (ER_COUNT_PAIRS | ER_PREC_FP32 | ER_PREC_COMP))
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
            ER_SYNC(ctx, ctx->stream);
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
            ER_SYNC(ctx, ctx->stream);
        } else {
            // D2H as float (half the bytes), widen on the host
            float* tmp = (float*)out;  // the first half of the caller's double buffer
            ER_CUDA(ctx, cudaMemcpyAsync(tmp, dst, npts * sizeof(float), cudaMemcpyDeviceToHost,
                                         ctx->stream));
            ER_SYNC(ctx, ctx->stream);
            double* o = (double*)out;
            for (size_t i = npts; i-- > 0;) o[i] = (double)tmp[i];
        }
    }
    return ER_OK;
}

int er_grid_sheet(er_ctx* ctx, int fw_id, int nx, int ny, int nz, int x_index,
                  double* out_sheet) {
    if (!ctx || !out_sheet) return ER_ERR_INVALID;
    if (int st = check_grid_dims(ctx, nx, ny, nz, "sheet")) return st;
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
    ER_SYNC(ctx, ctx->stream);
    const float* src = (const float*)ctx->pinned.ptr;
    for (size_t i = 0; i < ns; ++i) out_sheet[i] = (double)src[i];
    return ER_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batches
struct er_batch_plan {
    er_ctx* ctx = nullptr;
    int mode = ER_BATCH_PERSISTENT;
    int prec = 0;                  // er::PREC_NEAR64 (default) or er::PREC_COMP
    int n_jobs = 0;
    std::vector<GridTask> tasks;   // job order
    std::vector<int> order;        // queue position -> job (longest first)
    void* d_block = nullptr;       // one pool allocation: tasks, start, head
    GridTask* d_tasks = nullptr;   // queue order
    int* d_start = nullptr;        // n_jobs + 1 brick offsets, queue order
    int* d_head = nullptr;
    int n_items = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
};

namespace er {

// Queue order of the jobs, largest key first. For device output the key is
// the cost per brick (atoms per A^3: denser frameworks have more pairs per
// point), so the tail of the persistent queue holds the cheap bricks. For host
// output it is the grid size: a grid's copy to the host starts when its last
// brick is done, so the big grids go first and the copies left after the
// kernel ends are the small ones. (A brick is at most about half a
// millisecond of one CTA's work, so either order leaves a short kernel tail.)
static void queue_order(const std::vector<double>& cost, std::vector<int>& order) {
    order.resize(cost.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
}

static int plan_enqueue(er_batch_plan* p) {
    er_ctx* ctx = p->ctx;
    if (p->mode == ER_BATCH_PLAIN) {
        for (int i = 0; i < p->n_jobs; ++i) {
            int st = launch_grid_plain(ctx, p->tasks[i], p->prec);
            if (st != ER_OK) return st;
        }
        return ER_OK;
    }
    return launch_grid_persistent(ctx, p->d_tasks, p->d_start, p->n_jobs, p->n_items, p->d_head,
                                  p->prec);
}

}  // namespace er

extern "C" {

}  // extern "C"

namespace er {

// Builds a plan; with capture, the launch sequence is also captured as a graph
// (er_batch_plan_run replays it).
int plan_create(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode, bool capture,
                er_batch_plan** out, bool host_order = false) {
    if (!ctx || !out || (n_jobs > 0 && !jobs) || n_jobs < 0) return ER_ERR_INVALID;
    const bool autotune = (mode & ER_BATCH_AUTOTUNE) != 0;
    const int prec = (mode & ER_BATCH_COMP) ? PREC_COMP : PREC_NEAR64;
    mode &= ~(ER_BATCH_AUTOTUNE | ER_BATCH_COMP);
    if (mode != ER_BATCH_PERSISTENT && mode != ER_BATCH_PLAIN) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    *out = nullptr;
    er_batch_plan* p = new er_batch_plan();
    p->ctx = ctx;
    p->mode = mode;
    p->prec = prec;
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
            st = tune_tile(ctx, *f, jobs[i].nx, jobs[i].ny, jobs[i].nz, jobs[i].out_device, prec,
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
        cost.push_back(host_order ? (double)jobs[i].nx * jobs[i].ny * jobs[i].nz
                                  : (double)f->dev.n_img / std::max(1.0, f->volume));
    }
    queue_order(cost, p->order);
    auto fail = [&](int st, const char* m) {
        er_batch_plan_destroy(p);
        return set_error(ctx, st, m);
    };
    // queue-ordered tasks and brick offsets, staged in pinned memory, one copy
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t s_tasks = al(std::max(n_jobs, 1) * sizeof(GridTask));
    const size_t s_start = al((size_t)(n_jobs + 1) * sizeof(int));
    const size_t total = s_tasks + s_start + sizeof(int);
    if (ctx->plan_pinned.ensure(total) != ER_OK)
        return fail(ER_ERR_NOMEM, "batch: pinned staging failed");
    char* h = (char*)ctx->plan_pinned.ptr;
    GridTask* ht = (GridTask*)h;
    int* hs = (int*)(h + s_tasks);
    int64_t acc = 0;
    for (int q = 0; q < n_jobs; ++q) {
        ht[q] = p->tasks[p->order[q]];
        hs[q] = (int)acc;
        acc += task_bricks(ht[q]);
        if (acc > INT32_MAX) return fail(ER_ERR_LIMIT, "batch: more than 2^31 bricks");
    }
    hs[n_jobs] = (int)acc;
    p->n_items = (int)acc;
    if (pool_alloc(ctx, &p->d_block, total) != ER_OK)
        return fail(ER_ERR_NOMEM, "batch: device allocation failed");
    p->d_tasks = (GridTask*)p->d_block;
    p->d_start = (int*)((char*)p->d_block + s_tasks);
    p->d_head = (int*)((char*)p->d_block + s_tasks + s_start);
    if (cudaMemcpyAsync(p->d_block, h, s_tasks + s_start, cudaMemcpyHostToDevice, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(ER_ERR_CUDA, "batch: queue upload failed");
    }
    if (!capture) {
        *out = p;
        return ER_OK;
    }
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

}  // namespace er

extern "C" {

int er_batch_plan_create(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode,
                         er_batch_plan** out) {
    return plan_create(ctx, jobs, n_jobs, mode, true, out);
}

int er_batch_plan_run(er_batch_plan* p) {
    er::NvtxRange nvtx("er_batch_plan_run");
    if (p && !p->exec) return ER_ERR_INVALID;
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
    if (p->d_block) cudaFreeAsync(p->d_block, p->ctx->stream);
    delete p;
}

int er_grid_batch(er_ctx* ctx, const er_grid_job* jobs, int n_jobs, int mode) {
    er::NvtxRange nvtx("er_grid_batch");
    if (!ctx || n_jobs < 0 || (n_jobs > 0 && !jobs)) return ER_ERR_INVALID;
    if (mode & ER_BATCH_HOST_OUT) {
        // stage every grid in one device buffer; copy each back as soon as
        // the persistent kernel reports its last brick done
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
        const int inner = mode & ~ER_BATCH_HOST_OUT;
        auto copy_out = [&](int i) {
            return cudaMemcpyAsync(jobs[i].out_device, base + off[i],
                                   (off[i + 1] - off[i]) * sizeof(float), cudaMemcpyDeviceToHost,
                                   ctx->copy_stream);
        };
        if ((inner & ~(ER_BATCH_AUTOTUNE | ER_BATCH_COMP)) != ER_BATCH_PERSISTENT ||
            n_jobs == 0) {
            int st = er_grid_batch(ctx, dj.data(), n_jobs, inner);
            if (st != ER_OK) return st;
            for (int i = 0; i < n_jobs; ++i) ER_CUDA(ctx, copy_out(i));
            ER_CUDA(ctx, cudaStreamSynchronize(ctx->copy_stream));
            return ER_OK;
        }
        er_batch_plan* p = nullptr;
        int st = plan_create(ctx, dj.data(), n_jobs, inner, false, &p, true);
        if (st != ER_OK) return st;
        std::unique_ptr<er_batch_plan, void (*)(er_batch_plan*)> guard(p, er_batch_plan_destroy);
        // bricks left per queue position, and the host-visible flags
        std::vector<int> left(n_jobs);
        for (int q = 0; q < n_jobs; ++q) left[q] = (int)task_bricks(p->tasks[p->order[q]]);
        if (ctx->task_left.ensure((size_t)n_jobs * sizeof(int)) != ER_OK)
            return set_error(ctx, ER_ERR_NOMEM, "batch: device allocation failed");
        if (ctx->done_cap < (size_t)n_jobs) {
            if (ctx->done_host) cudaFreeHost(ctx->done_host);
            ctx->done_host = ctx->done_dev = nullptr;
            ctx->done_cap = 0;
            void* hp = nullptr;
            if (cudaHostAlloc(&hp, (size_t)n_jobs * sizeof(int), cudaHostAllocMapped) !=
                cudaSuccess) {
                cudaGetLastError();
                return set_error(ctx, ER_ERR_NOMEM, "batch: mapped flag allocation failed");
            }
            void* dp = nullptr;
            ER_CUDA(ctx, cudaHostGetDevicePointer(&dp, hp, 0));
            ctx->done_host = (int*)hp;
            ctx->done_dev = (int*)dp;
            ctx->done_cap = (size_t)n_jobs;
        }
        volatile int* done = ctx->done_host;
        for (int i = 0; i < n_jobs; ++i) done[i] = 0;
        int* d_left = (int*)ctx->task_left.ptr;
        ER_CUDA(ctx, cudaMemcpyAsync(d_left, left.data(), (size_t)n_jobs * sizeof(int),
                                     cudaMemcpyHostToDevice, ctx->stream));
        st = launch_grid_persistent(ctx, p->d_tasks, p->d_start, n_jobs, p->n_items, p->d_head,
                                    p->prec, d_left, ctx->done_dev);
        if (st != ER_OK) return st;
        cudaEvent_t fin;
        ER_CUDA(ctx, cudaEventCreateWithFlags(&fin, cudaEventDisableTiming));
        cudaError_t e = cudaEventRecord(fin, ctx->stream);
        std::vector<char> sent(n_jobs, 0);
        int n_sent = 0;
        // Poll until every grid is on its way; bounded by the kernel, which
        // has no device-side waits and so always finishes.
        while (e == cudaSuccess && n_sent < n_jobs) {
            const cudaError_t q = cudaEventQuery(fin);
            if (q != cudaSuccess && q != cudaErrorNotReady) {
                e = q;
                break;
            }
            const bool all = q == cudaSuccess;
            for (int k = 0; k < n_jobs && e == cudaSuccess; ++k)
                if (!sent[k] && (all || done[k])) {
                    e = copy_out(p->order[k]);
                    sent[k] = 1;
                    ++n_sent;
                }
            if (!all && n_sent < n_jobs) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
        cudaEventDestroy(fin);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->copy_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_error(ctx, e, "batch: run / copy-out");
        return take_fault(ctx);
    }
    er_batch_plan* p = nullptr;
    int st = er_batch_plan_create(ctx, jobs, n_jobs, mode, &p);
    if (st != ER_OK) return st;
    st = er_batch_plan_run(p);
    if (st == ER_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        st = cuda_error(ctx, cudaGetLastError(), "batch: run");
    if (st == ER_OK) st = take_fault(ctx);
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

// Largest |1 - x y0| over `per_thread` samples per thread of y0 =
// rcp.approx.ftz.f64(x), x = m 2^k with m uniform in [1, 2) (Philox stream 7)
// and k in [-80, 20) (the squared distances the near pairs can see). The
// residual is formed by one FMA, exact up to its final rounding.
__global__ void __launch_bounds__(256) rcp64_seed_kernel(int per_thread,
                                                         unsigned long long* max_bits) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double worst = 0.0;
    for (int i = 0; i < per_thread; ++i) {
        double f[3];
        insertion_point(7, tid * (uint64_t)per_thread + (uint64_t)i, f);
        const int k = (int)(f[1] * 100.0) - 80;
        const double x = ldexp(1.0 + f[0], k);
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
        worst = fmax(worst, fabs(fma(-x, y, 1.0)));
    }
    atomicMax(max_bits, (unsigned long long)__double_as_longlong(worst));
}

extern "C" int er_probe_rcp64_seed(er_ctx* ctx, double* max_rel_err) {
    if (!ctx || !max_rel_err) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->counter.ensure(4096 * sizeof(float)) != ER_OK)
        return set_error(ctx, ER_ERR_NOMEM, "probe: allocation failed");
    unsigned long long* bits = (unsigned long long*)ctx->counter.ptr;
    ER_CUDA(ctx, cudaMemsetAsync(bits, 0, sizeof(*bits), ctx->stream));
    rcp64_seed_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(64, bits);
    ER_CUDA(ctx, cudaGetLastError());
    unsigned long long h = 0;
    ER_CUDA(ctx, cudaMemcpyAsync(&h, bits, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    ER_SYNC(ctx, ctx->stream);
    double v;
    memcpy(&v, &h, sizeof(v));
    *max_rel_err = v;
    return ER_OK;
}

// One CTA waits, with the engine's bounded wait, for an mbarrier phase that
// nothing completes (no arrival, no copy); when the wait gives up it raises
// the fault word of `fault` as the engine's staging waits do.
__global__ void wait_timeout_kernel(int spins, int* fault) {
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool gave_up = !mbar_wait(&bar, 0u, spins);
    if (__syncthreads_or(gave_up) && threadIdx.x == 0) {
        atomicExch(fault, 1);
        mbar_inval(&bar);
    }
}

extern "C" int er_selftest_wait_timeout(er_ctx* ctx, int spins) {
    if (!ctx || spins < 1) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    if (int st = take_fault(ctx)) return st;  // an earlier fault is reported first
    wait_timeout_kernel<<<1, 64, 0, ctx->stream>>>(spins, ctx->fault_dev);
    ER_CUDA(ctx, cudaGetLastError());
    ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (take_fault(ctx) == ER_OK)
        return set_error(ctx, ER_ERR_CUDA, "selftest: the bounded wait did not report");
    return ER_OK;
}

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
