// er_noalloc.cu -- er_henry_stats_noalloc: Widom statistics that allocate nothing.
//
// Some callers cannot call cudaMalloc: a code whose device memory is carved
// up in advance by its own pool allocator (for example a Monte Carlo engine
// that sizes its pool at start-up and owns every byte), or a loop that cannot
// afford the implicit device-wide synchronisation and unbounded latency that
// cudaMalloc / cudaFree may bring. They still want the insertion-averaged
// Boltzmann factor of energies they already hold on the device. This entry
// point reduces such an energy array with the same FP64 log-sum-exp tree as
// er_henry, and keeps its only scratch -- one partial (m, s, se, n_inf,
// n_bad) per reduction block plus the final one, 4097 x 40 bytes -- in a
// file-scope static device array that every GPU loading this library holds
// until the process exits. Each call writes every slot it later reads, so
// nothing has to be cleared between calls; two calls that run at the same
// time on one GPU share the array and race. Index arithmetic is 64-bit, so
// every n up to ER_HENRY_STATS_NOALLOC_MAX_N partitions without overflow.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "er_ctx.h"

namespace er {
namespace noalloc {

struct Stats {
    double m, s, se;
    double n_inf;  // energies equal to +inf (weight 0), e.g. blocked insertions
    double n_bad;  // NaN or -inf energies: no defined weight, the call fails
};

// Reduction blocks; the static array holds kSlots partials plus the result.
constexpr int kSlots = 4096;

static __device__ __align__(256) Stats g_scratch[kSlots + 1];

__device__ __forceinline__ Stats merge(Stats a, Stats b) {
    const double ninf = a.n_inf + b.n_inf, nbad = a.n_bad + b.n_bad;
    if (b.s == 0.0) return Stats{a.m, a.s, a.se, ninf, nbad};
    if (a.s == 0.0) return Stats{b.m, b.s, b.se, ninf, nbad};
    const double M = fmax(a.m, b.m);
    const double fa = exp(a.m - M), fb = exp(b.m - M);
    return Stats{M, a.s * fa + b.s * fb, a.se * fa + b.se * fb, ninf, nbad};
}

__device__ __forceinline__ Stats tree(Stats v, Stats* sm) {
    const int t = threadIdx.x;
    sm[t] = v;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if (t < o) sm[t] = merge(sm[t], sm[t + o]);
        __syncthreads();
    }
    return sm[0];
}

// Block b reduces energies [b*chunk, (b+1)*chunk) in a fixed order and writes
// its triple to scratch[b]; every slot it will read later is written first.
__global__ void __launch_bounds__(256) partial_kernel(const float* __restrict__ E, int64_t n,
                                                      double T, int64_t chunk,
                                                      Stats* __restrict__ scratch) {
    __shared__ Stats sm[256];
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = lo + chunk < n ? lo + chunk : n;
    // two passes over this thread's entries, as er_henry's reduction: the
    // counts and the largest exponent, then the weights exp(x - m)
    Stats acc{-INFINITY, 0.0, 0.0, 0.0, 0.0};
    for (int64_t i = lo + threadIdx.x; i < hi; i += 256) {
        const float ef = E[i];
        if (ef == INFINITY) {  // +inf (a blocked insertion) has weight 0
            acc.n_inf += 1.0;
        } else if (isnan(ef) || ef == -INFINITY) {  // no defined weight
            acc.n_bad += 1.0;
        } else {
            acc.m = fmax(acc.m, -(double)ef / T);
        }
    }
    if (acc.m > -INFINITY) {
        for (int64_t i = lo + threadIdx.x; i < hi; i += 256) {
            const float ef = E[i];
            if (isinf(ef) || isnan(ef)) continue;
            const double e = (double)ef;
            const double w = exp(-e / T - acc.m);
            acc.s += w;
            acc.se += e * w;
        }
    }
    const Stats r = tree(acc, sm);
    if (threadIdx.x == 0) scratch[blockIdx.x] = r;
}

__global__ void __launch_bounds__(256) final_kernel(Stats* __restrict__ scratch, int nb) {
    __shared__ Stats sm[256];
    Stats acc{-INFINITY, 0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += 256) acc = merge(acc, scratch[i]);
    const Stats r = tree(acc, sm);
    if (threadIdx.x == 0) scratch[kSlots] = r;
}

// Device address of g_scratch per device ordinal, looked up once per device
// (with that device current) on the first call made on it.
constexpr int kMaxDevices = 64;
static Stats* g_scratch_addr[kMaxDevices] = {nullptr};
static std::mutex g_scratch_mu;

static int scratch_for(er_ctx* ctx, Stats** out) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return set_error(ctx, ER_ERR_LIMIT, "henry_stats_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[ctx->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_error(ctx, ER_ERR_CUDA,
                             std::string("henry_stats_noalloc: cudaGetSymbolAddress failed: ") +
                                 cudaGetErrorString(e));
        }
        g_scratch_addr[ctx->device] = (Stats*)p;
    }
    *out = g_scratch_addr[ctx->device];
    return ER_OK;
}

}  // namespace noalloc
}  // namespace er

using namespace er;

extern "C" int er_henry_stats_noalloc(er_ctx* ctx, const float* energies, int64_t n,
                                      double temperature, er_henry_result* out) {
    if (!ctx || !energies || !out) return ER_ERR_INVALID;
    if (n < 1 || n > ER_HENRY_STATS_NOALLOC_MAX_N)
        return set_error(ctx, ER_ERR_LIMIT,
                         "henry_stats_noalloc: n must be in [1, ER_HENRY_STATS_NOALLOC_MAX_N]");
    if (!(temperature > 0.0) || !std::isfinite(temperature))
        return set_error(ctx, ER_ERR_INVALID, "henry_stats_noalloc: temperature must be positive");
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    noalloc::Stats* scratch = nullptr;
    int st = noalloc::scratch_for(ctx, &scratch);
    if (st != ER_OK) return st;
    // the block partition of er_henry's reduction (4 blocks per SM, at most
    // kSlots), computed in 64-bit so that it cannot overflow at the top of the range
    const int64_t rblocks = std::min<int64_t>(noalloc::kSlots, std::max(1, ctx->num_sms * 4));
    const int64_t chunk = (n + rblocks - 1) / rblocks;
    const int nrb = (int)((n + chunk - 1) / chunk);
    noalloc::partial_kernel<<<nrb, 256, 0, ctx->stream>>>(energies, n, temperature, chunk,
                                                           scratch);
    noalloc::final_kernel<<<1, 256, 0, ctx->stream>>>(scratch, nrb);
    ER_CUDA(ctx, cudaGetLastError());
    noalloc::Stats r;
    ER_CUDA(ctx, cudaMemcpyAsync(&r, scratch + noalloc::kSlots, sizeof(r), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    ER_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (r.n_bad > 0.0)
        return set_error(ctx, ER_ERR_INVALID,
                         "henry_stats_noalloc: " + std::to_string((long long)r.n_bad) +
                             " energies are NaN or -inf");
    out->log_scale = r.m;
    out->sum_w_scaled = r.s;
    out->sum_ew_scaled = r.se;
    out->sum_w = r.s > 0 ? r.s * exp(r.m) : 0.0;
    out->sum_ew = r.s > 0 ? r.se * exp(r.m) : 0.0;
    out->n_insertions = (double)n;
    out->n_blocked = r.n_inf;
    out->mean_energy = r.s > 0 ? r.se / r.s : 0.0;
    out->kh_mol_m3_pa = out->sum_w / (double)n / temperature / 8.314;
    return ER_OK;
}
