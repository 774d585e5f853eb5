// er_build.cu -- the image cell lists of er_framework_upload_many, built on
// the device.
//
// What is built is the host build's (er_host.cc build_framework): every atom
// image a + n (n in [-rep, rep]^3, the image loop of
// src/computegridsheet.h:54-56) whose fractional overshoot of a slab times the
// slab width stays below the keep distance, at the Cartesian position r * f of
// the positioning frame, sorted into cells of edge h over the bounding box of
// the kept images, x index fastest, images of one cell in ascending image id.
// The device evaluates the same FP64 expressions in the same order, each
// operation rounded once (no contraction), so the blocks equal the host
// build's bit for bit.
//
// Only the atoms travel (position, sig2, FP64 and FP32 coefficients: 56 bytes
// per atom instead of ~44 bytes per kept image):
//   host:   validate and derive the per-atom arrays (all threads), one copy;
//   pass 1: one thread per candidate image: kept count and bounding box per
//           framework (block-reduced, one atomic per block and quantity);
//   host:   cell grid, block layout and allocation per framework;
//   pass 2: per group of frameworks: cell counts, exclusive scan, cell_start,
//           scatter into the cells, sort of each cell by image id (the
//           scatter's atomics leave the order inside a cell undefined), and
//           the per-atom arrays.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <string>
#include <vector>

#include "er_ctx.h"
#include "er_host.h"

namespace er {

namespace {

constexpr int kBuildThreads = 256;
// Pass-2 group limits: cells (count and scan arrays of one group) and images.
constexpr int64_t kGroupCells = (int64_t)1 << 26;
constexpr int64_t kGroupImages = (int64_t)INT32_MAX - 1;

struct BuildFw {
    double r[9];          // positioning frame (row-major)
    double w[3];          // perpendicular widths
    double keep;          // image-keep distance (A)
    double lo[3];         // cell grid corner (pass 2)
    double inv_h;         // 1 / cell edge
    long long cand;       // candidate images n_atoms * ipa
    int blk0;             // first candidate block of this framework
    int atom0;            // first atom in the per-atom arrays
    int n_atoms, ipa;
    int rep[3];
    int nc[3];            // cells per axis (pass 2)
    int cell0;            // first cell in its group's count array (pass 2)
    double4* img_xyz;     // destination block arrays (pass 2)
    float2* img_par;
    uint32_t* img_id;
    int* cell_start;
    double4* atom_frac;
    double2* atom_lj64;
    double2* img_lj64;
};

__device__ __forceinline__ unsigned long long order_key(double x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

double key_value(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
}

// Largest f in [lo, hi) with key(f) <= v (key non-decreasing, key(lo) <= v).
template <class K>
__device__ __forceinline__ int find_fw(int lo, int hi, long long v, K key) {
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (key(mid) <= v) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double overshoot(double f) {
    return f < 0 ? -f : (f > 1 ? __dsub_rn(f, 1.0) : 0.0);
}

// Candidate q of framework F: whether it is kept, and then its position.
__device__ __forceinline__ bool image_of(const BuildFw& F, const double4* __restrict__ af,
                                         const float2* __restrict__ ap, long long q, double& x,
                                         double& y, double& z, float2& par, int* atom = nullptr) {
    const int a = (int)(q / F.ipa);
    if (atom) *atom = a;
    const int code = (int)(q - (long long)a * F.ipa);
    par = ap[F.atom0 + a];
    if (par.x == 0.0f) return false;  // eps == 0 or sig == 0: no images
    const int ny = 2 * F.rep[1] + 1, nz = 2 * F.rep[2] + 1;
    const int i = code / (ny * nz) - F.rep[0];
    const int j = (code / nz) % ny - F.rep[1];
    const int k = code % nz - F.rep[2];
    const double4 p = af[F.atom0 + a];
    const double fx = __dadd_rn(p.x, (double)i);
    const double fy = __dadd_rn(p.y, (double)j);
    const double fz = __dadd_rn(p.z, (double)k);
    if (__dmul_rn(overshoot(fx), F.w[0]) >= F.keep || __dmul_rn(overshoot(fy), F.w[1]) >= F.keep ||
        __dmul_rn(overshoot(fz), F.w[2]) >= F.keep)
        return false;
    const double* t = F.r;
    x = __dadd_rn(__dadd_rn(__dmul_rn(t[0], fx), __dmul_rn(t[1], fy)), __dmul_rn(t[2], fz));
    y = __dadd_rn(__dadd_rn(__dmul_rn(t[3], fx), __dmul_rn(t[4], fy)), __dmul_rn(t[5], fz));
    z = __dadd_rn(__dadd_rn(__dmul_rn(t[6], fx), __dmul_rn(t[7], fy)), __dmul_rn(t[8], fz));
    return true;
}

__device__ __forceinline__ int cell_of(const BuildFw& F, double x, double y, double z) {
    const double v[3] = {x, y, z};
    int c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        c[k] = (int)floor(__dmul_rn(__dsub_rn(v[k], F.lo[k]), F.inv_h));
        c[k] = min(max(c[k], 0), F.nc[k] - 1);
    }
    return (c[2] * F.nc[1] + c[1]) * F.nc[0] + c[0];
}

// The framework and candidate index of this thread: blocks of one framework
// are contiguous (blk0), so a block never spans two frameworks.
__device__ __forceinline__ int block_fw(const int* __restrict__ blk0, int g0, int g1, int b) {
    return find_fw(g0, g1, b, [&](int m) { return (long long)blk0[m]; });
}

// Pass 1: kept images per framework and their bounding box (order keys).
__global__ void __launch_bounds__(kBuildThreads)
    build_count_kernel(const BuildFw* __restrict__ fws, const int* __restrict__ blk0, int n_fw,
                       const double4* __restrict__ af, const float2* __restrict__ ap,
                       unsigned* __restrict__ cnt, unsigned long long* __restrict__ lo,
                       unsigned long long* __restrict__ hi) {
    __shared__ unsigned long long red[kBuildThreads / 32][6];
    const int f = block_fw(blk0, 0, n_fw, blockIdx.x);
    const BuildFw& F = fws[f];
    const long long q = (long long)(blockIdx.x - blk0[f]) * kBuildThreads + threadIdx.x;
    double x = 0, y = 0, z = 0;
    float2 par;
    const bool kept = q < F.cand && image_of(F, af, ap, q, x, y, z, par);
    unsigned long long k[6];
    k[0] = kept ? order_key(x) : ~0ull;
    k[1] = kept ? order_key(y) : ~0ull;
    k[2] = kept ? order_key(z) : ~0ull;
    k[3] = kept ? order_key(x) : 0ull;
    k[4] = kept ? order_key(y) : 0ull;
    k[5] = kept ? order_key(z) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const unsigned long long a = __shfl_xor_sync(0xffffffffu, k[d], o);
            const unsigned long long b = __shfl_xor_sync(0xffffffffu, k[3 + d], o);
            k[d] = a < k[d] ? a : k[d];
            k[3 + d] = b > k[3 + d] ? b : k[3 + d];
        }
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int d = 0; d < 6; ++d) red[w][d] = k[d];
    const int n_kept = __syncthreads_count(kept);
    if (threadIdx.x == 0 && n_kept > 0) {
        for (int v = 1; v < kBuildThreads / 32; ++v)
            for (int d = 0; d < 3; ++d) {
                k[d] = red[v][d] < k[d] ? red[v][d] : k[d];
                k[3 + d] = red[v][3 + d] > k[3 + d] ? red[v][3 + d] : k[3 + d];
            }
        atomicAdd(&cnt[f], (unsigned)n_kept);
        for (int d = 0; d < 3; ++d) {
            atomicMin(&lo[3 * f + d], k[d]);
            atomicMax(&hi[3 * f + d], k[3 + d]);
        }
    }
}

// Pass 2a: images per cell.
__global__ void __launch_bounds__(kBuildThreads)
    build_cells_kernel(const BuildFw* __restrict__ fws, const int* __restrict__ blk0, int g0,
                       int g1, const double4* __restrict__ af, const float2* __restrict__ ap,
                       int* __restrict__ counts) {
    const int b = blk0[g0] + blockIdx.x;
    const int f = block_fw(blk0, g0, g1, b);
    const BuildFw& F = fws[f];
    const long long q = (long long)(b - blk0[f]) * kBuildThreads + threadIdx.x;
    double x, y, z;
    float2 par;
    if (q < F.cand && image_of(F, af, ap, q, x, y, z, par))
        atomicAdd(&counts[F.cell0 + cell_of(F, x, y, z)], 1);
}

// Pass 2b: cell_start of every framework of the group from the group scan
// (ncell + 1 entries per framework, framework m's first at cell0 + m - g0).
__global__ void build_starts_kernel(const BuildFw* __restrict__ fws, int g0, int g1, int n_entries,
                                    const int* __restrict__ starts) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_entries;
         i += gridDim.x * blockDim.x) {
        const int f = find_fw(g0, g1, i, [&](int m) { return (long long)fws[m].cell0 + (m - g0); });
        const BuildFw& F = fws[f];
        const int c = i - (F.cell0 + (f - g0));
        F.cell_start[c] = starts[F.cell0 + c] - starts[F.cell0];
    }
}

// Pass 2c: every kept image into its cell (order inside a cell undefined).
__global__ void __launch_bounds__(kBuildThreads)
    build_scatter_kernel(const BuildFw* __restrict__ fws, const int* __restrict__ blk0, int g0,
                         int g1, const double4* __restrict__ af, const float2* __restrict__ ap,
                         const double2* __restrict__ lj, int* __restrict__ fill) {
    const int b = blk0[g0] + blockIdx.x;
    const int f = block_fw(blk0, g0, g1, b);
    const BuildFw& F = fws[f];
    const long long q = (long long)(b - blk0[f]) * kBuildThreads + threadIdx.x;
    double x, y, z;
    float2 par;
    int a = 0;
    if (q < F.cand && image_of(F, af, ap, q, x, y, z, par, &a)) {
        const int c = cell_of(F, x, y, z);
        const int dst = F.cell_start[c] + atomicAdd(&fill[F.cell0 + c], 1);
        F.img_xyz[dst] = make_double4(x, y, z, 0.0);
        F.img_par[dst] = par;
        F.img_id[dst] = (uint32_t)q;
        F.img_lj64[dst] = lj[F.atom0 + a];
    }
}

// Pass 2d: each cell's images in ascending id (the host build's stable order).
__global__ void build_sort_kernel(const BuildFw* __restrict__ fws, int g0, int g1, int n_cells) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cells;
         i += gridDim.x * blockDim.x) {
        const int f = find_fw(g0, g1, i, [&](int m) { return (long long)fws[m].cell0; });
        const BuildFw& F = fws[f];
        const int c = i - F.cell0;
        const int b = F.cell_start[c], e = F.cell_start[c + 1];
        for (int u = b + 1; u < e; ++u) {
            const uint32_t id = F.img_id[u];
            const double4 p = F.img_xyz[u];
            const float2 pr = F.img_par[u];
            const double2 l = F.img_lj64[u];
            int v = u - 1;
            while (v >= b && F.img_id[v] > id) {
                F.img_id[v + 1] = F.img_id[v];
                F.img_xyz[v + 1] = F.img_xyz[v];
                F.img_par[v + 1] = F.img_par[v];
                F.img_lj64[v + 1] = F.img_lj64[v];
                --v;
            }
            F.img_id[v + 1] = id;
            F.img_xyz[v + 1] = p;
            F.img_par[v + 1] = pr;
            F.img_lj64[v + 1] = l;
        }
    }
}

// Pass 2e: the per-atom FP64 arrays into each block.
__global__ void build_atoms_kernel(const BuildFw* __restrict__ fws, int g0, int g1, int a0,
                                   int n_atoms, const double4* __restrict__ af,
                                   const double2* __restrict__ lj) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_atoms;
         i += gridDim.x * blockDim.x) {
        const int ga = a0 + i;
        const int f = find_fw(g0, g1, ga, [&](int m) { return (long long)fws[m].atom0; });
        const BuildFw& F = fws[f];
        F.atom_frac[ga - F.atom0] = af[ga];
        F.atom_lj64[ga - F.atom0] = lj[ga];
    }
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

unsigned grid_for(int64_t n) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
}

}  // namespace

int device_upload_many(er_ctx* ctx, const er_framework_desc* descs, int n, int* fw_ids) {
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const double h = ctx->cell_edge;
    // per-atom offsets
    std::vector<int64_t> atom0(n + 1, 0);
    for (int i = 0; i < n; ++i) atom0[i + 1] = atom0[i] + std::max(descs[i].n_atoms, 0);
    if (atom0[n] > INT32_MAX)
        return set_error(ctx, ER_ERR_LIMIT, "framework upload: more than 2^31 atoms in one call");
    const size_t A = (size_t)atom0[n];
    // staging layout (pinned and device copies alike)
    const size_t o_lj = al256(A * sizeof(double4));
    const size_t o_ap = o_lj + al256(A * sizeof(double2));
    const size_t o_fw = o_ap + al256(A * sizeof(float2));
    const size_t o_b0 = o_fw + al256((size_t)n * sizeof(BuildFw));
    const size_t s_up = o_b0 + al256((size_t)(n + 1) * sizeof(int));  // bytes copied up
    const size_t o_cnt = s_up;
    const size_t o_lo = o_cnt + al256((size_t)n * sizeof(unsigned));
    const size_t o_hi = o_lo + al256((size_t)3 * n * sizeof(unsigned long long));
    const size_t s_all = o_hi + al256((size_t)3 * n * sizeof(unsigned long long));
    if (ctx->pinned.ensure(s_all) != ER_OK)
        return set_error(ctx, ER_ERR_NOMEM, "framework upload: pinned staging failed");
    char* hp = (char*)ctx->pinned.ptr;
    HostImage* h_af = (HostImage*)hp;
    double* h_lj = (double*)(hp + o_lj);
    float* h_ap = (float*)(hp + o_ap);
    BuildFw* h_fw = (BuildFw*)(hp + o_fw);
    int* h_b0 = (int*)(hp + o_b0);
    unsigned* h_cnt = (unsigned*)(hp + o_cnt);
    unsigned long long* h_lo = (unsigned long long*)(hp + o_lo);
    unsigned long long* h_hi = (unsigned long long*)(hp + o_hi);

    // 1. validation and per-atom arrays, on the host threads
    std::vector<HostFramework> hfs(n);
    std::vector<std::string> errs(n);
    std::vector<int> sts(n, ER_OK);
    parallel_for(n, [&](int i) {
        double w[3] = {0, 0, 0}, keep = 0;
        const int64_t a0 = atom0[i];
        sts[i] = prepare_framework(descs[i], h, hfs[i], errs[i], h_af + a0, h_lj + 2 * a0,
                                   h_ap + 2 * a0, w, &keep);
        if (sts[i] != ER_OK) return;
        BuildFw& F = h_fw[i];
        memset(&F, 0, sizeof F);
        for (int k = 0; k < 9; ++k) F.r[k] = hfs[i].r[k];
        for (int k = 0; k < 3; ++k) {
            F.w[k] = w[k];
            F.rep[k] = hfs[i].rep[k];
        }
        F.keep = keep;
        F.ipa = hfs[i].imgs_per_atom;
        F.n_atoms = hfs[i].n_atoms;
        F.atom0 = (int)a0;
        F.cand = (long long)F.n_atoms * F.ipa;
        F.inv_h = 1.0 / h;
    });
    for (int i = 0; i < n; ++i)
        if (sts[i] != ER_OK)
            return set_error(ctx, sts[i],
                             n > 1 ? "framework " + std::to_string(i) + ": " + errs[i] : errs[i]);
    int64_t nblk = 0;
    for (int i = 0; i < n; ++i) {
        h_b0[i] = (int)nblk;
        h_fw[i].blk0 = (int)nblk;
        nblk += (h_fw[i].cand + kBuildThreads - 1) / kBuildThreads;
        if (nblk > INT32_MAX)
            return set_error(ctx, ER_ERR_LIMIT, "framework upload: too many candidate images");
    }
    h_b0[n] = (int)nblk;

    // 2. scratch, one copy up, pass 1, results down
    std::vector<void*> blocks(n, nullptr);
    void* scratch = nullptr;
    void* cells = nullptr;
    auto release = [&]() {
        cudaStreamSynchronize(st);
        for (void* b : blocks)
            if (b) cudaFreeAsync(b, st);
        if (scratch) cudaFreeAsync(scratch, st);
        if (cells) cudaFreeAsync(cells, st);
    };
    auto fail = [&](int status, const std::string& m) {
        release();
        return set_error(ctx, status, m);
    };
    auto fail_cuda = [&](cudaError_t e, const char* what) {
        release();
        return cuda_error(ctx, e, what);
    };
    if (pool_alloc(ctx, &scratch, s_all) != ER_OK)
        return fail(ER_ERR_NOMEM, "framework upload: device allocation failed");
    char* dp = (char*)scratch;
    const double4* d_af = (const double4*)dp;
    const double2* d_lj = (const double2*)(dp + o_lj);
    const float2* d_ap = (const float2*)(dp + o_ap);
    BuildFw* d_fw = (BuildFw*)(dp + o_fw);
    const int* d_b0 = (const int*)(dp + o_b0);
    unsigned* d_cnt = (unsigned*)(dp + o_cnt);
    unsigned long long* d_lo = (unsigned long long*)(dp + o_lo);
    unsigned long long* d_hi = (unsigned long long*)(dp + o_hi);
    cudaError_t e = cudaMemcpyAsync(dp, hp, s_up, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_cnt, 0, (size_t)n * sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_lo, 0xff, (size_t)3 * n * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_hi, 0, (size_t)3 * n * 8, st);
    if (e == cudaSuccess && nblk > 0) {
        build_count_kernel<<<(unsigned)nblk, kBuildThreads, 0, st>>>(d_fw, d_b0, n, d_af, d_ap,
                                                                     d_cnt, d_lo, d_hi);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hp + o_cnt, dp + o_cnt, s_all - o_cnt,
                                              cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(e, "framework upload: pass 1");

    // 3. cell grids, layouts and blocks
    std::vector<FwLayout> lay(n);
    std::vector<int64_t> ncell(n, 0);
    for (int i = 0; i < n; ++i) {
        const unsigned n_img = h_cnt[i];
        if ((size_t)n_img >= (size_t)INT32_MAX)
            return fail(ER_ERR_LIMIT, "framework " + std::to_string(i) + ": too many images");
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        if (n_img > 0)
            for (int k = 0; k < 3; ++k) {
                lo[k] = key_value(h_lo[3 * i + k]);
                hi[k] = key_value(h_hi[3 * i + k]);
            }
        std::string err;
        if (int s2 = cell_grid(lo, hi, h, hfs[i], &ncell[i], err))
            return fail(s2, n > 1 ? "framework " + std::to_string(i) + ": " + err : err);
        lay[i] = fw_layout(n_img, (size_t)ncell[i] + 1, (size_t)hfs[i].n_atoms);
        if (pool_alloc(ctx, &blocks[i], lay[i].total) != ER_OK)
            return fail(ER_ERR_NOMEM, "framework upload: device allocation failed");
        BuildFw& F = h_fw[i];
        char* b = (char*)blocks[i];
        for (int k = 0; k < 3; ++k) {
            F.lo[k] = hfs[i].cell_lo[k];
            F.nc[k] = hfs[i].nc[k];
        }
        F.img_xyz = (double4*)b;
        F.img_par = (float2*)(b + lay[i].o_par);
        F.img_id = (uint32_t*)(b + lay[i].o_id);
        F.cell_start = (int*)(b + lay[i].o_cs);
        F.atom_frac = (double4*)(b + lay[i].o_af);
        F.atom_lj64 = (double2*)(b + lay[i].o_lj);
        F.img_lj64 = (double2*)(b + lay[i].o_ilj);
    }
    // groups of frameworks whose cells and images fit one scan
    std::vector<int> gstart(1, 0);
    int64_t gc = 0, gi = 0, cmax = 0;
    for (int i = 0; i < n; ++i) {
        if (i > gstart.back() && (gc + ncell[i] > kGroupCells || gi + h_cnt[i] > kGroupImages)) {
            gstart.push_back(i);
            gc = gi = 0;
        }
        h_fw[i].cell0 = (int)gc;
        gc += ncell[i];
        gi += h_cnt[i];
        cmax = std::max(cmax, gc);
    }
    gstart.push_back(n);
    const size_t s_counts = al256((size_t)cmax * sizeof(int));
    const size_t s_starts = al256((size_t)(cmax + 1) * sizeof(int));
    const size_t s_tiles = al256((size_t)std::max(scan_tiles((int)cmax), 1) * sizeof(int));
    if (pool_alloc(ctx, &cells, s_counts + s_starts + s_tiles) != ER_OK)
        return fail(ER_ERR_NOMEM, "framework upload: device allocation failed");
    int* d_counts = (int*)cells;
    int* d_starts = (int*)((char*)cells + s_counts);
    int* d_tiles = (int*)((char*)cells + s_counts + s_starts);
    // the pass-1 copy up has completed (synchronised above): reuse its staging
    e = cudaMemcpyAsync(d_fw, h_fw, (size_t)n * sizeof(BuildFw), cudaMemcpyHostToDevice, st);

    // 4. pass 2, group by group
    for (size_t g = 0; g + 1 < gstart.size() && e == cudaSuccess; ++g) {
        const int g0 = gstart[g], g1 = gstart[g + 1];
        int64_t C = 0;
        for (int i = g0; i < g1; ++i) C += ncell[i];
        const int gblk = h_b0[g1] - h_b0[g0];
        e = cudaMemsetAsync(d_counts, 0, (size_t)C * sizeof(int), st);
        if (e != cudaSuccess) break;
        if (gblk > 0)
            build_cells_kernel<<<gblk, kBuildThreads, 0, st>>>(d_fw, d_b0, g0, g1, d_af, d_ap,
                                                               d_counts);
        if (int s2 = scan_exclusive(ctx, d_counts, (int)C, d_starts, d_tiles, st)) {
            release();
            return s2;
        }
        const int64_t n_entries = C + (g1 - g0);
        build_starts_kernel<<<grid_for(n_entries), 256, 0, st>>>(d_fw, g0, g1, (int)n_entries,
                                                                 d_starts);
        e = cudaMemsetAsync(d_counts, 0, (size_t)C * sizeof(int), st);
        if (e != cudaSuccess) break;
        if (gblk > 0)
            build_scatter_kernel<<<gblk, kBuildThreads, 0, st>>>(d_fw, d_b0, g0, g1, d_af, d_ap,
                                                                 d_lj, d_counts);
        build_sort_kernel<<<grid_for(C), 256, 0, st>>>(d_fw, g0, g1, (int)C);
        const int64_t ga = atom0[g1] - atom0[g0];
        if (ga > 0)
            build_atoms_kernel<<<grid_for(ga), 256, 0, st>>>(d_fw, g0, g1, (int)atom0[g0], (int)ga,
                                                             d_af, d_lj);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(e, "framework upload: pass 2");
    cudaFreeAsync(scratch, st);
    cudaFreeAsync(cells, st);
    for (int i = 0; i < n; ++i) {
        FwRecord rec;
        fw_record(hfs[i], h_cnt[i], lay[i], blocks[i], rec);
        rec.dev.fault = ctx->fault_dev;
        const int id = ctx->next_fw++;
        ctx->fws[id] = rec;
        fw_ids[i] = id;
    }
    return ER_OK;
}

}  // namespace er
