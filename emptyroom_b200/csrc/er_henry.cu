// er_henry.cu -- Widom insertions and the Henry coefficient (er_henry).
//
// Replaces doHenry (src/doHenry.h:29-135) and its host reduction
// (src/henry.cu:157-174). Pipeline, all on the context stream:
//   1. gen     insertion i -> Philox4x32-10 point (stream `seed`), pocket-mask
//              test, spatial bin key (bins of ~32 expected points, 2x2x2 bricks)
//   2. scan    bin counts -> bin starts
//   3. scatter insertion indices into their bins; 4. place each sorted
//      position's point, then order the bins that straddle a warp boundary by
//      insertion index (so every warp's point set, and with it every FP32
//      rounding, is deterministic)
//   5. energy  the shared LJ engine over 2048 (1024 for runs below 1e6)
//              points per CTA, in bin order
//   6. reduce  FP64 log-sum-exp of exp(-E/T) and E exp(-E/T) in insertion
//              order with a fixed tree: (m, s, se) with sum w = s e^m.
#include <math.h>

#include <climits>

#include <algorithm>

#include "er_ctx.h"
#include "er_nvtx.h"
#include "er_engine.cuh"
#include "er_philox.h"

namespace er {

// Insertions per thread of the energy kernel: 8 for large runs (1.82 against
// 2.00 ms per 1e7 insertions on a config-1 cell); 4 below kHenrySmallN, where
// a run fills few waves of CTAs and more, smaller CTAs finish sooner (0.16
// against 0.26 ms for 1e5 insertions).
constexpr int kHenryP = 8;
constexpr int kHenryPSmall = 4;
constexpr int64_t kHenrySmallN = 1000000;
inline int henry_points_per_thread(int64_t n) { return n < kHenrySmallN ? kHenryPSmall : kHenryP; }

struct BinGeom {
    int nb[3];  // bins per fractional axis
    int NB[3];  // 2x2x2 bricks per axis
    int n_keys;
};

struct Lse {
    double m, s, se;
};

// Bin of a point: bins grouped in 2x2x2 bricks, bricks in serpentine order
// (y runs backwards on odd x layers, z backwards on the odd rows of the
// traversal), so consecutive bricks are always face neighbours and any run of
// consecutive sorted points -- a warp's or a CTA's -- spans a compact box, also
// where it straddles the end of a brick row (plain row order would put the
// next brick at the far side of the cell there).
__device__ __forceinline__ int bin_key(const double* f, const BinGeom& g) {
    int b[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) b[d] = min(g.nb[d] - 1, max(0, (int)(f[d] * g.nb[d])));
    const int bx = b[0] >> 1;
    int by = b[1] >> 1, bz = b[2] >> 1;
    if (bx & 1) by = g.NB[1] - 1 - by;
    if ((bx * g.NB[1] + by) & 1) bz = g.NB[2] - 1 - bz;
    return ((bx * g.NB[1] + by) * g.NB[2] + bz) * 8 + ((b[0] & 1) << 2) + ((b[1] & 1) << 1) +
           (b[2] & 1);
}

// Pocket-mask geometry of a grid of nx x ny x nz points with axes i/(N-1):
// the spacings 1/(N-1) (FP64, the reference's dx, src/gcmc.cc:155-157) and
// N - 1, for the cell lookup below.
struct MaskGeom {
    int n[3];        // points per axis
    double d[3];     // 1/(N-1), rounded to nearest as the reference computes it
    double nm1[3];   // N - 1
};

// Cell index along one axis: floor(p / d) as src/gcmc.cc:155-157 computes
// it, clamped to N - 2. p * (N - 1) is within a few ulps of p / d, so their
// floors can differ only where the quotient lies within ~1e-12 of an integer;
// there the FP64 division itself decides.
__device__ __forceinline__ int mask_cell(double p, double d, double nm1, int n) {
    const double q = p * nm1;
    int c = (int)floor(q);
    if (fabs(q - rint(q)) < 1e-6) c = (int)floor(__ddiv_rn(p, d));
    return min(c, n - 2);
}

// cell[i, j, k] = 1 when any of the 8 grid points at the corners of the cell
// (i..i+1, j..j+1, k..k+1) is blocked, for i < nx - 1, j < ny - 1,
// k < nz - 1: an insertion in the cell is blocked exactly when the
// reference's lookup of its 8 surrounding grid energies meets a blocked one.
__global__ void mask_cells_kernel(const uint8_t* __restrict__ mask, MaskGeom mg,
                                  uint8_t* __restrict__ cell) {
    const int cx = mg.n[0] - 1, cy = mg.n[1] - 1, cz = mg.n[2] - 1;
    const size_t total = (size_t)cx * cy * cz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < total;
         c += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(c % cz);
        const int j = (int)((c / cz) % cy);
        const int i = (int)(c / ((size_t)cz * cy));
        uint8_t b = 0;
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj) {
                const size_t row =
                    (size_t)(j + dj) * mg.n[2] + (size_t)(i + di) * mg.n[1] * mg.n[2];
                b |= mask[row + k] | mask[row + k + 1];
            }
        cell[c] = b ? 1 : 0;
    }
}

// Insertion i: its point, the mask test, its bin key and its slot in the bin
// (the count before it; slots within a bin are in arbitrary order, which is
// made ascending where a bin straddles a warp boundary).
// The blocked test is one load from the cell mask (mask_cells_kernel).
__global__ void henry_gen_kernel(uint64_t seed, int n, BinGeom g,
                                 const uint8_t* __restrict__ cell, MaskGeom mg,
                                 int* __restrict__ key, int* __restrict__ slot,
                                 int* __restrict__ counts, float* __restrict__ energies,
                                 int* __restrict__ n_blocked) {
    // 64-bit stride: near the 2^31 - 4097 limit i + stride leaves int
    for (long long ii = blockIdx.x * (long long)blockDim.x + threadIdx.x; ii < n;
         ii += (long long)gridDim.x * blockDim.x) {
        const int i = (int)ii;
        double f[3];
        insertion_point(seed, (uint64_t)i, f);
        bool blocked = false;
        if (cell) {
            const int ci = mask_cell(f[0], mg.d[0], mg.nm1[0], mg.n[0]);
            const int cj = mask_cell(f[1], mg.d[1], mg.nm1[1], mg.n[1]);
            const int ck = mask_cell(f[2], mg.d[2], mg.nm1[2], mg.n[2]);
            blocked = cell[(size_t)ck + (size_t)cj * (mg.n[2] - 1) +
                           (size_t)ci * (mg.n[1] - 1) * (mg.n[2] - 1)] != 0;
        }
        if (blocked) {
            key[i] = -1;
            energies[i] = INFINITY;
            atomicAdd(n_blocked, 1);
        } else {
            const int k = bin_key(f, g);
            key[i] = k;
            slot[i] = atomicAdd(&counts[k], 1);
        }
    }
}

// Exclusive scan of n ints (the bin counts) in three coalesced passes over
// tiles of kScanTile: tile sums, a one-CTA scan of the tile sums, then each
// tile scanned on chip and offset; out[n] receives the total.
constexpr int kScanThreads = 256, kScanPer = 8, kScanTile = kScanThreads * kScanPer;

__device__ __forceinline__ int cta_exscan256(int v, int* wsum, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < kScanThreads / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < kScanThreads / 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kScanThreads / 32) wsum[lane] = t;
    }
    __syncthreads();
    const int base = w ? wsum[w - 1] : 0;
    *total = wsum[kScanThreads / 32 - 1];
    __syncthreads();
    return base + x - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(const int* __restrict__ in,
                                                                  int n, int* __restrict__ sums) {
    __shared__ int wsum[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int v = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t i = base + k * kScanThreads + threadIdx.x;
        if (i < n) v += in[i];
    }
    int tot;
    cta_exscan256(v, wsum, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) scan_top_kernel(int* __restrict__ sums, int n_tiles,
                                                        int* __restrict__ total_out) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int per = (n_tiles + 1023) / 1024;  // a few contiguous tile sums per thread
    const int lo = min(n_tiles, t * per), hi = min(n_tiles, lo + per);
    int s = 0;
    for (int i = lo; i < hi; ++i) s += sums[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int i = lo; i < hi; ++i) {
        const int v = sums[i];
        sums[i] = run;
        run += v;
    }
    if (t == 1023) *total_out = part[1023];
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const int* __restrict__ in,
                                                                  int n,
                                                                  const int* __restrict__ sums,
                                                                  int* __restrict__ out) {
    __shared__ int tile[kScanTile];
    __shared__ int wsum[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t i = base + k * kScanThreads + threadIdx.x;
        tile[k * kScanThreads + threadIdx.x] = i < n ? in[i] : 0;
    }
    __syncthreads();
    // each thread owns kScanPer consecutive entries of the tile
    int v[kScanPer], s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = tile[threadIdx.x * kScanPer + k];
        s += v[k];
    }
    int tot;
    int run = cta_exscan256(s, wsum, &tot) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        tile[threadIdx.x * kScanPer + k] = run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const int64_t i = base + k * kScanThreads + threadIdx.x;
        if (i < n) out[i] = tile[k * kScanThreads + threadIdx.x];
    }
}

int scan_tiles(int n) { return (n + kScanTile - 1) / kScanTile; }

int scan_exclusive(er_ctx* ctx, const int* in, int n, int* out, int* tile_sums,
                   cudaStream_t st) {
    if (n <= 0) {
        ER_CUDA(ctx, cudaMemsetAsync(out, 0, sizeof(int), st));
        return ER_OK;
    }
    const int tiles = scan_tiles(n);
    scan_tiles_kernel<<<tiles, kScanThreads, 0, st>>>(in, n, tile_sums);
    scan_top_kernel<<<1, 1024, 0, st>>>(tile_sums, tiles, out + n);
    scan_apply_kernel<<<tiles, kScanThreads, 0, st>>>(in, n, tile_sums, out);
    ER_CUDA(ctx, cudaGetLastError());
    return ER_OK;
}

// Four insertions per thread (16-byte loads of key and slot): their four
// bin-start lookups are in flight together (the kernel waits on those
// dependent loads; one insertion per thread took 0.108 ms per 1e7).
__global__ void henry_scatter_kernel(const int* __restrict__ key, const int* __restrict__ slot,
                                     int n, const int* __restrict__ starts,
                                     int* __restrict__ tmp) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; 4 * g < n;
         g += (long long)gridDim.x * blockDim.x) {
        const int i0 = (int)(4 * g);
        if (i0 + 4 <= n) {
            const int4 k = *reinterpret_cast<const int4*>(key + i0);
            const int4 q = *reinterpret_cast<const int4*>(slot + i0);
            const int s0 = k.x >= 0 ? starts[k.x] : 0, s1 = k.y >= 0 ? starts[k.y] : 0;
            const int s2 = k.z >= 0 ? starts[k.z] : 0, s3 = k.w >= 0 ? starts[k.w] : 0;
            if (k.x >= 0) tmp[s0 + q.x] = i0;
            if (k.y >= 0) tmp[s1 + q.y] = i0 + 1;
            if (k.z >= 0) tmp[s2 + q.z] = i0 + 2;
            if (k.w >= 0) tmp[s3 + q.w] = i0 + 3;
        } else {
            for (int i = i0; i < n; ++i) {
                const int k = key[i];
                if (k >= 0) tmp[starts[k] + slot[i]] = i;
            }
        }
    }
}

// The positioning frame r of a framework, by value.
struct Frame {
    double r[9];
};

// The energy kernel's result for an insertion depends only on the set of
// insertions in its warp (warp_pts consecutive sorted positions) and in its
// CTA, not on their order there: every sum is per point, over lists built from
// the warp and CTA boxes, and the exact cutoff corrections add up in list
// order. So a bin inside one warp's positions keeps the order of its atomic
// slots (which varies from run to run), and only a bin that straddles a warp
// boundary (one in eight at ~4 P points per bin) is put in ascending insertion
// order, which fixes the set on either side of the boundary. Sorting every bin
// (a warp per bin) took 0.33 ms per 1e7 insertions with the scatter; ordering
// only the straddling bins in that kernel 0.25 ms; a thread per position for
// the placement and a warp per boundary for the straddling bins 0.24 ms.
//
// The insertion point (recomputed from its Philox counter) is written at its
// position as its Cartesian position in frame r (the engine's own
// frac_to_cart, so the bits are those the engine would compute), which the
// energy kernel reads coalesced.
__device__ __forceinline__ void put_point(uint64_t seed, const Frame& fr, int v, double* dst) {
    double f[3], x, y, z;
    insertion_point(seed, (uint64_t)v, f);
    frac_to_cart(fr.r, f[0], f[1], f[2], x, y, z);
    dst[0] = x;
    dst[1] = y;
    dst[2] = z;
}

// Every sorted position p < n_valid, one thread each: the insertion the
// scatter put there and its point.
__global__ void henry_place_kernel(const int* __restrict__ n_valid, const int* __restrict__ tmp,
                                   uint64_t seed, Frame fr, int* __restrict__ order,
                                   double* __restrict__ pts) {
    const long long nv = *n_valid;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nv;
         p += (long long)gridDim.x * blockDim.x) {
        const int v = tmp[p];
        order[p] = v;
        put_point(seed, fr, v, pts + 3 * p);
    }
}

// One warp per warp boundary m * warp_pts (m >= 1) below n_valid, after
// henry_place_kernel: the bin holding that position (binary search of the bin
// starts); when the boundary cuts it and is the first boundary to do so, the
// warp rewrites the bin in ascending insertion order (each entry's rank among
// the bin's entries, compared 32 at a time through shuffles).
__global__ void henry_order_straddling_kernel(const int* __restrict__ starts, int n_keys,
                                              int warp_pts, const int* __restrict__ tmp,
                                              uint64_t seed, Frame fr, int* __restrict__ order,
                                              double* __restrict__ pts) {
    const int lane = threadIdx.x & 31;
    const long long m = ((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5) + 1;
    const long long qb = m * warp_pts;
    if (qb >= starts[n_keys]) return;
    const int q = (int)qb;
    // the last bin b with starts[b] <= q: q lies in [starts[b], starts[b + 1])
    int lo = 0, hi = n_keys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (starts[mid] <= q) lo = mid;
        else hi = mid - 1;
    }
    const int s = starts[lo], L = starts[lo + 1] - s;
    if (s == q || q - warp_pts > s) return;  // not cut here, or cut first by an earlier boundary
    for (int q0 = 0; q0 < L; q0 += 32) {
        const int i = q0 + lane;
        const int v = i < L ? tmp[s + i] : INT_MAX;
        int rank = 0;
        for (int r0 = 0; r0 < L; r0 += 32) {
            const int u = r0 + lane < L ? tmp[s + r0 + lane] : INT_MAX;
#pragma unroll
            for (int k = 0; k < 32; ++k) rank += __shfl_sync(0xffffffffu, u, k) < v;
        }
        if (i < L) {
            order[s + rank] = v;
            put_point(seed, fr, v, pts + 3 * (size_t)(s + rank));
        }
    }
}

template <int P>
__global__ void __launch_bounds__(kThreads, 2)
    henry_energy_kernel(const __grid_constant__ PointTask task) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    if ((long long)blockIdx.x * (kWarps * 32 * P) >= (long long)*task.n_valid) return;
    EngineSmem& s = *reinterpret_cast<EngineSmem*>(smem_raw);
    PointPolicy<P> pol(&task, blockIdx.x);
    // near pairs in FP64: a Boltzmann factor turns an energy error dE into a
    // relative weight error dE / T, so Widom energies get the tighter mode
    process_cta<PointPolicy<P>, PREC_NEAR64>(s, pol, task.fw, task.cc);
}

__device__ __forceinline__ Lse lse_merge(Lse a, Lse b) {
    if (b.s == 0.0) return a;
    if (a.s == 0.0) return b;
    const double M = fmax(a.m, b.m);
    const double fa = exp(a.m - M), fb = exp(b.m - M);
    return Lse{M, a.s * fa + b.s * fb, a.se * fa + b.se * fb};
}

__device__ __forceinline__ Lse lse_tree(Lse v, Lse* sm) {
    const int t = threadIdx.x;
    sm[t] = v;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
        if (t < o) sm[t] = lse_merge(sm[t], sm[t + o]);
        __syncthreads();
    }
    return sm[0];
}

// Block b sums insertions [b*chunk, (b+1)*chunk) (thread t: b*chunk + t + 256 k).
// neg_inv_t = -1 / T: the exponent -E / T of src/doHenry.h:107 as a product
// (within an ulp of the quotient; the Boltzmann factor moves by ~1e-15 relative).
__global__ void __launch_bounds__(256) henry_reduce_kernel(const float* __restrict__ E, int n,
                                                           double neg_inv_t, int chunk,
                                                           Lse* __restrict__ part) {
    __shared__ Lse sm[256];
    const int lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    // two passes over this thread's entries: the largest exponent, then the
    // weights exp(x - m), which do not wait for one another (with a running
    // maximum every exp waited for the previous one). x is the rounded product
    // in both passes (__dmul_rn: no FMA contraction into x - m), so the largest
    // entry's weight is exactly 1 also for capped energies, where |x| ~ 1e27.
    double m = -INFINITY;
    for (int i = lo + threadIdx.x; i < hi; i += 256) {
        const float ef = E[i];
        if (!isinf(ef)) m = fmax(m, __dmul_rn((double)ef, neg_inv_t));  // blocked: weight 0
    }
    Lse acc{m, 0.0, 0.0};
    if (m > -INFINITY) {
        for (int i = lo + threadIdx.x; i < hi; i += 256) {
            const float ef = E[i];
            if (isinf(ef)) continue;
            const double e = (double)ef;
            const double w = exp(__dmul_rn(e, neg_inv_t) - m);
            acc.s += w;
            acc.se += e * w;
        }
    }
    const Lse r = lse_tree(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void __launch_bounds__(256) henry_final_kernel(const Lse* __restrict__ part, int nb,
                                                          Lse* __restrict__ out) {
    __shared__ Lse sm[256];
    Lse acc{-INFINITY, 0.0, 0.0};
    for (int i = threadIdx.x; i < nb; i += 256) acc = lse_merge(acc, part[i]);
    const Lse r = lse_tree(acc, sm);
    if (threadIdx.x == 0) *out = r;
}


int henry_reserve(er_ctx* ctx, HenryScratch& hs, int64_t n, cudaStream_t st) {
    const size_t N = (size_t)n;
    cudaMemPool_t pool = ctx->pool;
    if (hs.pts.ensure_on(3 * N * sizeof(double), pool, st) ||
        hs.bin.ensure_on(N * sizeof(int), pool, st) ||
        hs.order.ensure_on(N * sizeof(int), pool, st) ||
        hs.tmp.ensure_on(N * sizeof(int), pool, st) || hs.e.ensure_on(N * sizeof(float), pool, st))
        return set_error(ctx, ER_ERR_NOMEM, "henry: device scratch allocation failed");
    return ER_OK;
}

int henry_enqueue(er_ctx* ctx, const FwRecord& fw, double temperature, int n, uint64_t seed,
                  const uint8_t* block_mask, int mnx, int mny, int mnz, cudaStream_t st,
                  HenryScratch& hs, HenryOut* host_out) {
    // bins of ~4 P expected points (a 2x2x2 brick of bins ~ one warp's 32 P
    // points), shaped after the cell vector lengths
    BinGeom g;
    {
        const double L0 = fw.cell_len[0], L1 = fw.cell_len[1], L2 = fw.cell_len[2];
        const double scale =
            cbrt((double)n / (4.0 * henry_points_per_thread(n)) / (L0 * L1 * L2));
        const double L[3] = {L0, L1, L2};
        int64_t nk = 8;
        for (int d = 0; d < 3; ++d) {
            g.nb[d] = (int)std::min<double>(2048.0, std::max(1.0, floor(L[d] * scale + 0.5)));
            g.NB[d] = (g.nb[d] + 1) / 2;
            nk *= g.NB[d];
        }
        if (nk > (int64_t)256 * 1024 * 1024)
            return set_error(ctx, ER_ERR_LIMIT, "henry: bin table too large");
        g.n_keys = (int)nk;
    }
    const size_t N = (size_t)n;
    // scratch grows in stream order from the context's pool (no device-wide
    // synchronisation while other streams run jobs)
    cudaMemPool_t pool = ctx->pool;
    if (hs.pts.ensure_on(3 * N * sizeof(double), pool, st) ||
        hs.bin.ensure_on(N * sizeof(int), pool, st) ||
        hs.order.ensure_on(N * sizeof(int), pool, st) ||
        hs.tmp.ensure_on(N * sizeof(int), pool, st) ||
        hs.counts.ensure_on(2 * (size_t)g.n_keys * sizeof(int), pool, st) ||
        hs.starts.ensure_on(((size_t)g.n_keys + 1) * sizeof(int), pool, st) ||
        hs.e.ensure_on(N * sizeof(float), pool, st) ||
        hs.nblk.ensure_on(4 * sizeof(int), pool, st) ||
        hs.part.ensure_on(4096 * sizeof(Lse), pool, st) ||
        hs.res.ensure_on(sizeof(Lse), pool, st))
        return set_error(ctx, ER_ERR_NOMEM, "henry: device scratch allocation failed");
    const uint8_t* d_mask = nullptr;
    if (block_mask) {
        cudaPointerAttributes attr;
        const bool on_device = cudaPointerGetAttributes(&attr, block_mask) == cudaSuccess &&
                               attr.type == cudaMemoryTypeDevice;
        cudaGetLastError();
        if (on_device) {
            d_mask = block_mask;  // e.g. the output of er_block_pockets_device
        } else {
            const size_t mb = (size_t)mnx * mny * mnz;
            if (hs.mask.ensure_on(mb, ctx->pool, st))
                return set_error(ctx, ER_ERR_NOMEM, "henry: mask allocation");
            ER_CUDA(ctx, cudaMemcpyAsync(hs.mask.ptr, block_mask, mb, cudaMemcpyHostToDevice, st));
            d_mask = (const uint8_t*)hs.mask.ptr;
        }
    }
    int* counts = (int*)hs.counts.ptr;
    int* tsum = counts + g.n_keys;  // tile sums of the scan
    int* starts = (int*)hs.starts.ptr;
    int* nblk = (int*)hs.nblk.ptr;
    float* E = (float*)hs.e.ptr;
    ER_CUDA(ctx, cudaMemsetAsync(counts, 0, (size_t)g.n_keys * sizeof(int), st));
    ER_CUDA(ctx, cudaMemsetAsync(nblk, 0, sizeof(int), st));
    const int gthreads = 256;
    const int gblocks = (int)std::min<int64_t>((n + gthreads - 1) / gthreads,
                                               (int64_t)ctx->num_sms * 32);
    // the slot of each insertion in its bin goes to `order` until the sort
    // overwrites it with the sorted insertion indices
    int* slot = (int*)hs.order.ptr;
    if (hs.ev[0]) ER_CUDA(ctx, cudaEventRecord(hs.ev[0], st));
    MaskGeom mg{};
    const uint8_t* d_cell = nullptr;
    if (d_mask) {
        const int dims[3] = {mnx, mny, mnz};
        for (int k = 0; k < 3; ++k) {
            mg.n[k] = dims[k];
            mg.d[k] = 1.0 / (double)(dims[k] - 1);
            mg.nm1[k] = (double)(dims[k] - 1);
        }
        const size_t nc = (size_t)(mnx - 1) * (mny - 1) * (mnz - 1);
        if (hs.cell.ensure_on(nc, ctx->pool, st))
            return set_error(ctx, ER_ERR_NOMEM, "henry: cell mask allocation");
        const int cb = (int)std::min<size_t>((nc + 255) / 256, (size_t)ctx->num_sms * 16);
        mask_cells_kernel<<<cb, 256, 0, st>>>(d_mask, mg, (uint8_t*)hs.cell.ptr);
        d_cell = (const uint8_t*)hs.cell.ptr;
    }
    henry_gen_kernel<<<gblocks, gthreads, 0, st>>>(seed, n, g, d_cell, mg, (int*)hs.bin.ptr, slot,
                                                   counts, E, nblk);
    {
        const int tiles = (g.n_keys + kScanTile - 1) / kScanTile;
        scan_tiles_kernel<<<tiles, kScanThreads, 0, st>>>(counts, g.n_keys, tsum);
        scan_top_kernel<<<1, 1024, 0, st>>>(tsum, tiles, starts + g.n_keys);
        scan_apply_kernel<<<tiles, kScanThreads, 0, st>>>(counts, g.n_keys, tsum, starts);
    }
    if (hs.ev[0]) ER_CUDA(ctx, cudaEventRecord(hs.ev[1], st));
    // a thread per four insertions for the scatter and a thread per position
    // for the placement, up to 2^20 CTAs each (more blocks in flight hide their
    // dependent loads; key and slot are pool allocations, 16-byte aligned);
    // a warp per warp boundary for the straddling bins
    const int sblocks = (int)std::min<int64_t>(((int64_t)n + 4 * gthreads - 1) / (4 * gthreads),
                                               1 << 20);
    const int pblocks = (int)std::min<int64_t>(((int64_t)n + gthreads - 1) / gthreads, 1 << 20);
    henry_scatter_kernel<<<sblocks, gthreads, 0, st>>>((const int*)hs.bin.ptr, slot, n, starts,
                                                       (int*)hs.tmp.ptr);
    Frame fr;
    for (int k = 0; k < 9; ++k) fr.r[k] = fw.dev.r[k];
    henry_place_kernel<<<pblocks, gthreads, 0, st>>>(starts + g.n_keys, (const int*)hs.tmp.ptr,
                                                      seed, fr, (int*)hs.order.ptr,
                                                      (double*)hs.pts.ptr);
    const int warp_pts = 32 * henry_points_per_thread(n);
    const int64_t n_bounds = ((int64_t)n - 1) / warp_pts;  // boundaries below n
    if (n_bounds > 0)
        henry_order_straddling_kernel<<<(int)((n_bounds + 7) / 8), 256, 0, st>>>(
            starts, g.n_keys, warp_pts, (const int*)hs.tmp.ptr, seed, fr, (int*)hs.order.ptr,
            (double*)hs.pts.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    if (hs.ev[0]) ER_CUDA(ctx, cudaEventRecord(hs.ev[2], st));
    PointTask task;
    task.fw = fw.dev;
    task.cc = make_cutoff_consts(fw.rc2, 0.0, 1e-16 * 1e-16);  // min_r, src/doHenry.h:15
    task.pts = (const double*)hs.pts.ptr;
    task.order = (const int*)hs.order.ptr;
    task.seed = seed;
    task.n_valid = starts + g.n_keys;
    task.energies = E;
    const int hp = henry_points_per_thread(n);
    const int per_cta = kWarps * 32 * hp;
    const int ecta = (n + per_cta - 1) / per_cta;
    if (hp == kHenryP) {
        ER_CUDA(ctx, cudaFuncSetAttribute(henry_energy_kernel<kHenryP>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(EngineSmem)));
        henry_energy_kernel<kHenryP><<<ecta, kThreads, sizeof(EngineSmem), st>>>(task);
    } else {
        ER_CUDA(ctx, cudaFuncSetAttribute(henry_energy_kernel<kHenryPSmall>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(EngineSmem)));
        henry_energy_kernel<kHenryPSmall><<<ecta, kThreads, sizeof(EngineSmem), st>>>(task);
    }
    ER_CUDA(ctx, cudaGetLastError());
    if (hs.ev[0]) ER_CUDA(ctx, cudaEventRecord(hs.ev[3], st));
    const int rblocks = std::min(4096, std::max(1, ctx->num_sms * 4));
    const int chunk = (n + rblocks - 1) / rblocks;
    const int nrb = (n + chunk - 1) / chunk;
    henry_reduce_kernel<<<nrb, 256, 0, st>>>(E, n, -1.0 / temperature, chunk, (Lse*)hs.part.ptr);
    henry_final_kernel<<<1, 256, 0, st>>>((const Lse*)hs.part.ptr, nrb, (Lse*)hs.res.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    if (hs.ev[0]) ER_CUDA(ctx, cudaEventRecord(hs.ev[4], st));
    if (host_out) {
        ER_CUDA(ctx, cudaMemcpyAsync(host_out->lse, hs.res.ptr, sizeof(Lse),
                                     cudaMemcpyDeviceToHost, st));
        ER_CUDA(ctx, cudaMemcpyAsync(&host_out->n_blocked, nblk, sizeof(int),
                                     cudaMemcpyDeviceToHost, st));
    }
    return ER_OK;
}

void henry_finish(const HenryOut& h, int64_t n, double temperature, er_henry_result* out) {
    const double m = h.lse[0], s = h.lse[1], se = h.lse[2];
    out->log_scale = m;
    out->sum_w_scaled = s;
    out->sum_ew_scaled = se;
    out->sum_w = s > 0 ? s * exp(m) : 0.0;
    out->sum_ew = s > 0 ? se * exp(m) : 0.0;
    out->n_insertions = (double)n;
    out->n_blocked = (double)h.n_blocked;
    out->mean_energy = s > 0 ? se / s : 0.0;
    // K_H = sum w / N / T / 8.314 (mol/(m^3 Pa)), src/henry.cu:169
    out->kh_mol_m3_pa = out->sum_w / (double)n / temperature / 8.314;
}

int henry_check(er_ctx* ctx, double temperature, int64_t n_ins, const uint8_t* block_mask,
                int mnx, int mny, int mnz) {
    if (!(temperature > 0.0) || !std::isfinite(temperature))
        return set_error(ctx, ER_ERR_INVALID, "henry: temperature must be positive");
    if (n_ins < 1) return set_error(ctx, ER_ERR_INVALID, "henry: n_ins must be >= 1");
    if (n_ins > (int64_t)INT32_MAX - 4096)
        return set_error(ctx, ER_ERR_LIMIT, "henry: more than 2^31 - 4097 insertions per call");
    if (block_mask && (mnx < 2 || mny < 2 || mnz < 2))
        return set_error(ctx, ER_ERR_INVALID, "henry: mask dims must be >= 2");
    return ER_OK;
}

}  // namespace er

using namespace er;

extern "C" int er_henry(er_ctx* ctx, int fw_id, double temperature, int64_t n_ins, uint64_t seed,
                        const uint8_t* block_mask, int mnx, int mny, int mnz,
                        er_henry_result* out, float* energies_out) {
    er::NvtxRange nvtx("er_henry");
    if (!ctx || !out) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    const FwRecord* f = find_fw(ctx, fw_id);
    if (!f) return set_error(ctx, ER_ERR_NOT_FOUND, "henry: unknown framework id");
    int st = henry_check(ctx, temperature, n_ins, block_mask, mnx, mny, mnz);
    if (st != ER_OK) return st;
    HenryOut h;
    st = henry_enqueue(ctx, *f, temperature, (int)n_ins, seed, block_mask, mnx, mny, mnz,
                       ctx->stream, ctx->henry, &h);
    if (st != ER_OK) return st;
    if (energies_out)
        ER_CUDA(ctx, cudaMemcpyAsync(energies_out, ctx->henry.e.ptr, (size_t)n_ins * sizeof(float),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    ER_SYNC(ctx, ctx->stream);
    henry_finish(h, n_ins, temperature, out);
    return ER_OK;
}

extern "C" int er_ctx_set_timing(er_ctx* ctx, int on) {
    if (!ctx) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    HenryScratch& hs = ctx->henry;
    if (on && !hs.ev[0]) {
        cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
        for (cudaEvent_t& e : ev) {
            const cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) {
                for (cudaEvent_t& x : ev)
                    if (x) cudaEventDestroy(x);
                return cuda_error(ctx, err, "henry timing: cudaEventCreate");
            }
        }
        for (int k = 0; k < 5; ++k) hs.ev[k] = ev[k];
    } else if (!on && hs.ev[0]) {
        ER_SYNC(ctx, ctx->stream);
        for (cudaEvent_t& e : hs.ev) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    }
    return ER_OK;
}

extern "C" int er_henry_last_timing(er_ctx* ctx, er_henry_timing* out) {
    if (!ctx || !out) return ER_ERR_INVALID;
    *out = er_henry_timing{0.0, 0.0, 0.0, 0.0};
    const HenryScratch& hs = ctx->henry;
    if (!hs.ev[0]) return set_error(ctx, ER_ERR_INVALID, "henry timing: timing is off");
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    float ms[4];
    for (int k = 0; k < 4; ++k) {
        const cudaError_t e = cudaEventElapsedTime(&ms[k], hs.ev[k], hs.ev[k + 1]);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(ctx, ER_ERR_INVALID, "henry timing: no timed er_henry call yet");
        }
    }
    *out = er_henry_timing{ms[0], ms[1], ms[2], ms[3]};
    return ER_OK;
}

// ------------------------------------------------------------------ Widom batch
// er_henry_batch: frameworks handed out to kHenryPipes pipelines, each a host
// thread driving its own stream and scratch (HenryPipe), so that one
// framework's grid, pocket labelling, binning and host round trips run while
// another's energy kernel holds the SMs. Every step is the single-call code
// (fill_grid_task + the plain grid kernel as er_grid, block_pockets_device_on
// as er_block_pockets_device, henry_enqueue as er_henry), so each result
// equals the single calls' bit for bit.
namespace er {
namespace {

// Up to 6 pipelines: on 64 config-4 frameworks (1e7 insertions, 80^3 pocket
// grids) 2, 3, 4 and 6 took 136.0, 133.8, 132.6 and 130.7 ms. Each holds its
// own scratch, so the count is also cut to what half the free device memory
// holds (henry_pipe_count).
constexpr int kHenryPipes = 6;

// Device bytes one pipeline holds for a job: 40 per insertion (Cartesian
// FP64 point, bin key, order, scan scratch, FP32 energy), 24 per blocking-grid
// point (FP32 grid, mask, pocket labels and segments), plus the bin tables.
size_t henry_pipe_bytes(int64_t n_ins, const int bd[3]) {
    return 40 * (size_t)n_ins + 24 * (size_t)bd[0] * bd[1] * bd[2] + ((size_t)64 << 20);
}

int henry_pipe_count(er_ctx* ctx, int n, int64_t n_ins, const int bd[3]) {
    int np = std::min(n, kHenryPipes);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    // memory the pool keeps for reuse, and the pipelines' own scratch, count
    // as free: a new job grows into them first
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) ==
            cudaSuccess &&
        cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
        free_b += (size_t)(reserved - used);
    else
        cudaGetLastError();
    for (int p = 0; p < np && p < (int)ctx->pipes.size(); ++p) {
        const HenryPipe& P = *ctx->pipes[p];
        free_b += P.hs.bytes() + P.grid.cap + P.mask.cap;
    }
    const size_t fit = free_b / 2 / henry_pipe_bytes(n_ins, bd);
    return (int)std::max<size_t>(1, std::min<size_t>(np, fit));
}

int henry_one(er_ctx* ctx, HenryPipe& P, const FwRecord& fw, double temperature, int64_t n_ins,
              uint64_t seed, const int bd[3], er_henry_result* out, int* n_pockets) {
    const cudaStream_t st = P.stream;
    const uint8_t* mask = nullptr;
    int npk = 0;
    if (bd[0]) {
        const size_t pts = (size_t)bd[0] * bd[1] * bd[2];
        if (P.grid.ensure_on(pts * sizeof(float), ctx->pool, st) ||
            P.mask.ensure_on(pts, ctx->pool, st))
            return set_error(ctx, ER_ERR_NOMEM, "henry batch: grid/mask allocation failed");
        GridTask t;
        int s = fill_grid_task(ctx, fw, bd[0], bd[1], bd[2], (float*)P.grid.ptr, t, 4);
        if (s == ER_OK) s = launch_grid_plain_on(ctx, t, PREC_NEAR64, st);
        if (s == ER_OK)
            s = block_pockets_device_on(ctx, P.ps, st, (const float*)P.grid.ptr, bd[0], bd[1],
                                        bd[2], temperature, (uint8_t*)P.mask.ptr, &npk);
        if (s != ER_OK) return s;
        mask = (const uint8_t*)P.mask.ptr;
    }
    int s = henry_enqueue(ctx, fw, temperature, (int)n_ins, seed, mask, bd[0], bd[1], bd[2], st,
                          P.hs, P.out);
    if (s != ER_OK) return s;
    ER_SYNC(ctx, st);
    henry_finish(*P.out, n_ins, temperature, out);
    if (n_pockets) *n_pockets = npk;
    return ER_OK;
}

}  // namespace
}  // namespace er

extern "C" int er_henry_batch(er_ctx* ctx, const int* fw_ids, int n, double temperature,
                              int64_t n_insertions, const uint64_t* seeds, int block_nx,
                              int block_ny, int block_nz, er_henry_result* results,
                              int* n_pockets) {
    er::NvtxRange nvtx("er_henry_batch");
    if (!ctx || n < 0 || (n > 0 && (!fw_ids || !seeds || !results))) return ER_ERR_INVALID;
    if (n == 0) return ER_OK;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    int st = henry_check(ctx, temperature, n_insertions, nullptr, 0, 0, 0);
    if (st != ER_OK) return st;
    const bool blocking = block_nx != 0 || block_ny != 0 || block_nz != 0;
    const int bd[3] = {blocking ? block_nx : 0, blocking ? block_ny : 0, blocking ? block_nz : 0};
    if (blocking) {
        if ((st = check_grid_dims(ctx, block_nx, block_ny, block_nz, "henry batch")) != ER_OK)
            return st;
        if ((int64_t)block_nx * block_ny * block_nz >= (int64_t)INT32_MAX)
            return set_error(ctx, ER_ERR_LIMIT, "henry batch: blocking grid must have < 2^31 points");
    }
    std::vector<const FwRecord*> fr(n);
    for (int k = 0; k < n; ++k)
        if (!(fr[k] = find_fw(ctx, fw_ids[k])))
            return set_error(ctx, ER_ERR_NOT_FOUND,
                             "henry batch: unknown framework id (entry " + std::to_string(k) + ")");
    const int np = henry_pipe_count(ctx, n, n_insertions, bd);
    while ((int)ctx->pipes.size() < np) {
        HenryPipe* p = new HenryPipe();
        if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaMallocHost((void**)&p->out, sizeof(HenryOut)) != cudaSuccess) {
            cudaGetLastError();
            if (p->stream) cudaStreamDestroy(p->stream);
            delete p;
            return set_error(ctx, ER_ERR_CUDA, "henry batch: stream creation failed");
        }
        ctx->pipes.push_back(p);
    }
    // the pipelines' scratch and the framework blocks come from the pool in
    // stream order: order every pipeline after the work already queued
    cudaEvent_t ready;
    ER_CUDA(ctx, cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    ER_CUDA(ctx, cudaEventRecord(ready, ctx->stream));
    for (int p = 0; p < np; ++p) ER_CUDA(ctx, cudaStreamWaitEvent(ctx->pipes[p]->stream, ready, 0));
    cudaEventDestroy(ready);
    std::atomic<int> next(0), stop(0);
    std::vector<int> status(np, ER_OK);
    auto work = [&](int p) {
        if (cudaSetDevice(ctx->device) != cudaSuccess) {
            status[p] = set_error(ctx, ER_ERR_CUDA, "henry batch: cudaSetDevice failed");
            stop = 1;
            return;
        }
        for (int k; !stop && (k = next.fetch_add(1)) < n;) {
            const int s = henry_one(ctx, *ctx->pipes[p], *fr[k], temperature, n_insertions,
                                    seeds[k], bd, &results[k], n_pockets ? &n_pockets[k] : nullptr);
            if (s != ER_OK) {
                status[p] = s;
                stop = 1;
                return;
            }
        }
    };
    std::vector<std::thread> th;
    for (int p = 1; p < np; ++p) th.emplace_back(work, p);
    work(0);
    for (auto& t : th) t.join();
    for (int p = 0; p < np; ++p) {
        cudaStreamSynchronize(ctx->pipes[p]->stream);
        if (status[p] != ER_OK) return status[p];
    }
    return take_fault(ctx);
}
