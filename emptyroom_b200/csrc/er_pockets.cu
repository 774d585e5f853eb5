// er_pockets.cu -- pocket blocking on the GPU (er_block_pockets*) and the
// hard-sphere accessibility grid (er_accessibility).
//
// FindAndBlockPockets (src/pocketblocking.cc:126-391) labels 6-connected
// segments of accessible points (E < 15 T) with a serial flood fill in scan
// order, links segments across the three periodic faces, and calls a segment
// a POCKET unless a walk over those links returns to it in another unit cell.
// Here:
//   1. init      label[p] = p for accessible points, -1 otherwise
//   2. union     lock-free union-find over the -x, -y, -z neighbours, first
//                inside 4 x 8 x 32-point tiles in shared memory, then across
//                the tile faces in global memory; a root is always linked to
//                a smaller root, so every component ends rooted at its
//                smallest linear index
//   3. compress  label[p] = root
//   4. number    roots ranked in index order (device-wide scan) -- the
//                reference's segment numbers, since its flood fill meets each
//                segment first at the segment's smallest index
//   5. faces     links (from = segment at N-1, to = segment at 0, direction),
//                deduplicated in a device hash set
//   6. classify  on the host: weighted union-find over the (few) links; a
//                component is a CHANNEL iff some link contradicts the unit-cell
//                offsets (a cycle with non-zero net translation, self-links
//                included) -- the same verdict as the reference's DFS, which
//                checks every link of the component against a spanning walk
//   7. block     pocket points -> 1e13 (host double grid) or mask = 1 (device)
#include <math.h>

#include <algorithm>
#include <vector>

#include "er_ctx.h"
#include "er_nvtx.h"

namespace er {

__global__ void cc_init_f64(const double* __restrict__ E, int64_t n, double thr,
                            int* __restrict__ lab) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        lab[p] = (E[p] >= thr) ? -1 : (int)p;  // src/pocketblocking.cc:138
}

__global__ void cc_init_f32(const float* __restrict__ E, int64_t n, double thr,
                            int* __restrict__ lab) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        lab[p] = ((double)E[p] >= thr) ? -1 : (int)p;
}

__device__ __forceinline__ int cc_find(const int* lab, int x) {
    int y = lab[x];
    while (y != x) {
        x = y;
        y = lab[x];
    }
    return x;
}

// The same walk reading through L2 (labels change under concurrent unions).
// Labels only ever decrease along a chain, so the walk ends.
__device__ __forceinline__ int cc_find_l2(const int* lab, int x) {
    int y = __ldcg(lab + x);
    while (y != x) {
        x = y;
        y = __ldcg(lab + x);
    }
    return x;
}

// Links the roots of a and b (larger root under smaller). Every failed CAS
// means another thread has just linked that root to a smaller label, so a
// strictly decreases and the loop ends.
__device__ __forceinline__ void cc_unite(int* lab, int a, int b) {
    for (;;) {
        a = cc_find_l2(lab, a);
        b = cc_find_l2(lab, b);
        if (a == b) return;
        if (a < b) {
            const int t = a; a = b; b = t;
        }
        const int old = atomicCAS(&lab[a], a, b);
        if (old == a) return;
        a = old;
    }
}

// Tiled labelling: a CTA labels one tile of kTI x kTJ x kTK points (k fastest,
// so a warp reads 32 consecutive points) by union-find in shared memory, then
// writes each accessible point's label as the global index of its tile-local
// root. Local indices order like global ones inside a tile, and a tile-local
// root is the smallest index of its local component, so every label is <= its
// point and roots point to themselves: a valid state for cc_unite. The unions
// across tile faces follow in cc_union_faces, after every tile has written
// (a face union into a tile that had not yet written could be overwritten).
// Against one grid-wide union pass with global atomics: 0.38 -> 0.26 ms for
// the device pocket mask of a 129^3 grid (block_pockets_device, host-timed).
constexpr int kTK = 32, kTJ = 8, kTI = 4, kTile = kTK * kTJ * kTI;

__device__ __forceinline__ int cc_find_s(const int* sl, int x) {
    int y = sl[x];
    while (y != x) {
        x = y;
        y = sl[x];
    }
    return x;
}

__device__ __forceinline__ void cc_unite_s(int* sl, int a, int b) {
    for (;;) {
        a = cc_find_s(sl, a);
        b = cc_find_s(sl, b);
        if (a == b) return;
        if (a < b) {
            const int t = a; a = b; b = t;
        }
        const int old = atomicCAS(&sl[a], a, b);
        if (old == a) return;
        a = old;
    }
}

__global__ void __launch_bounds__(256) cc_union_tiles(int* __restrict__ lab, int nx, int ny,
                                                      int nz) {
    __shared__ int sl[kTile];
    const int tk = (nz + kTK - 1) / kTK, tj = (ny + kTJ - 1) / kTJ;
    const int k0 = (blockIdx.x % tk) * kTK;
    const int j0 = ((blockIdx.x / tk) % tj) * kTJ;
    const int i0 = (blockIdx.x / (tk * tj)) * kTI;
    const int64_t syz = (int64_t)ny * nz;
    auto gidx = [&](int q, bool& in) -> int64_t {
        const int lk = q % kTK, lj = (q / kTK) % kTJ, li = q / (kTK * kTJ);
        const int i = i0 + li, j = j0 + lj, k = k0 + lk;
        in = i < nx && j < ny && k < nz;
        return (int64_t)k + (int64_t)j * nz + (int64_t)i * syz;
    };
    for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
        bool in;
        const int64_t g = gidx(q, in);
        sl[q] = (in && lab[g] >= 0) ? q : -1;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
        if (sl[q] < 0) continue;
        const int lk = q % kTK, lj = (q / kTK) % kTJ, li = q / (kTK * kTJ);
        if (lk > 0 && sl[q - 1] >= 0) cc_unite_s(sl, q, q - 1);
        if (lj > 0 && sl[q - kTK] >= 0) cc_unite_s(sl, q, q - kTK);
        if (li > 0 && sl[q - kTK * kTJ] >= 0) cc_unite_s(sl, q, q - kTK * kTJ);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
        if (sl[q] < 0) continue;
        bool in;
        const int64_t g = gidx(q, in);
        lab[g] = (int)gidx(cc_find_s(sl, q), in);
    }
}

// Unions across the lower faces of the tiles (global union-find).
__global__ void cc_union_faces(int* __restrict__ lab, int nx, int ny, int nz) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t syz = (int64_t)ny * nz;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(p % nz);
        const int j = (int)((p / nz) % ny);
        const int i = (int)(p / syz);
        const bool fk = k > 0 && k % kTK == 0, fj = j > 0 && j % kTJ == 0;
        const bool fi = i > 0 && i % kTI == 0;
        if (!(fk || fj || fi) || lab[p] < 0) continue;
        if (fk && lab[p - 1] >= 0) cc_unite(lab, (int)p, (int)(p - 1));
        if (fj && lab[p - nz] >= 0) cc_unite(lab, (int)p, (int)(p - nz));
        if (fi && lab[p - syz] >= 0) cc_unite(lab, (int)p, (int)(p - syz));
    }
}

__global__ void cc_compress(int* __restrict__ lab, int64_t n) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        if (lab[p] >= 0) lab[p] = cc_find(lab, (int)p);
    }
}

constexpr int kScanItems = 4096;  // points per scan block (1024 threads x 4)

// Number of roots in each block of kScanItems points.
__global__ void __launch_bounds__(1024) cc_root_counts(const int* __restrict__ lab, int64_t n,
                                                       int* __restrict__ counts) {
    const int64_t base = (int64_t)blockIdx.x * kScanItems;
    int c = 0;
    for (int q = threadIdx.x; q < kScanItems; q += 1024) {
        const int64_t p = base + q;
        if (p < n && lab[p] == (int)p) ++c;
    }
    __shared__ int s[32];
    int v = c;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        int w = s[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) counts[blockIdx.x] = w;
    }
}

// Exclusive scan of n ints by one CTA (contiguous chunks); out[n] = total.
__global__ void __launch_bounds__(1024) cc_scan_small(const int* __restrict__ in,
                                                      int* __restrict__ out, int n) {
    __shared__ int sums[1024];
    const int t = threadIdx.x;
    const int per = (n + 1023) / 1024;
    const int lo = min(n, t * per), hi = min(n, lo + per);
    int s = 0;
    for (int i = lo; i < hi; ++i) s += in[i];
    sums[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = t >= o ? sums[t - o] : 0;
        __syncthreads();
        sums[t] += v;
        __syncthreads();
    }
    int run = sums[t] - s;
    for (int i = lo; i < hi; ++i) {
        const int v = in[i];
        out[i] = run;
        run += v;
    }
    if (t == 1023) out[n] = sums[1023];
}

// rank[p] = number of roots below p, for every root p (thread q owns points
// base + 4q .. base + 4q + 3, so ranks follow the linear index).
__global__ void __launch_bounds__(1024) cc_root_ranks(const int* __restrict__ lab, int64_t n,
                                                      const int* __restrict__ block_off,
                                                      int* __restrict__ rank) {
    __shared__ int wsum[32];
    const int64_t base = (int64_t)blockIdx.x * kScanItems + 4 * threadIdx.x;
    int f[4], c = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int64_t p = base + u;
        f[u] = (p < n && lab[p] == (int)p) ? 1 : 0;
        c += f[u];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;
    }
    __syncthreads();
    int run = block_off[blockIdx.x] + (w ? wsum[w - 1] : 0) + x - c;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        if (f[u]) rank[base + u] = run;
        run += f[u];
    }
}

__global__ void cc_segments(const int* __restrict__ lab, const int* __restrict__ rank, int64_t n,
                            int* __restrict__ seg) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int l = lab[p];
        seg[p] = l >= 0 ? rank[l] : -1;
    }
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// Face links of src/pocketblocking.cc:277-321, inserted once each into an
// open-addressing set; new keys are appended to `list`.
__global__ void cc_face_links(const int* __restrict__ seg, int nx, int ny, int nz,
                              unsigned long long* __restrict__ table, int table_mask,
                              unsigned long long* __restrict__ list, int* __restrict__ n_list,
                              int list_cap) {
    const int64_t fx = (int64_t)ny * nz, fy = (int64_t)nx * nz, fz = (int64_t)nx * ny;
    const int64_t total = fx + fy + fz;
    const int64_t syz = (int64_t)ny * nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        int64_t a, b;
        int dir;
        if (q < fx) {  // i = 0 face against i = N_x - 1
            const int j = (int)(q / nz), k = (int)(q % nz);
            a = (int64_t)k + (int64_t)j * nz;
            b = a + (int64_t)(nx - 1) * syz;
            dir = 1;
        } else if (q < fx + fy) {  // j = 0 face against j = N_y - 1
            const int64_t r = q - fx;
            const int i = (int)(r / nz), k = (int)(r % nz);
            a = (int64_t)k + (int64_t)i * syz;
            b = a + (int64_t)(ny - 1) * nz;
            dir = 2;
        } else {  // k = 0 face against k = N_z - 1
            const int64_t r = q - fx - fy;
            const int i = (int)(r / ny), j = (int)(r % ny);
            a = (int64_t)j * nz + (int64_t)i * syz;
            b = a + (nz - 1);
            dir = 3;
        }
        const int to = seg[a], from = seg[b];
        if (to < 0 || from < 0) continue;
        const unsigned long long key = ((unsigned long long)from << 34) |
                                       ((unsigned long long)to << 4) | (unsigned long long)dir;
        unsigned h = (unsigned)(mix64(key) & (uint64_t)table_mask);
        for (int probe = 0; probe <= table_mask; ++probe) {
            const unsigned long long old = atomicCAS(&table[h], ~0ull, key);
            if (old == ~0ull) {
                const int at = atomicAdd(n_list, 1);
                if (at < list_cap) list[at] = key;
                break;
            }
            if (old == key) break;
            h = (h + 1) & (unsigned)table_mask;
        }
    }
}

__global__ void cc_block_f64(double* __restrict__ E, const int* __restrict__ seg, int64_t n,
                             const unsigned char* __restrict__ pocket) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int s = seg[p];
        if (s >= 0 && pocket[s]) E[p] = 1e13;  // src/pocketblocking.cc:373-382
    }
}

__global__ void cc_block_mask(uint8_t* __restrict__ mask, const int* __restrict__ seg, int64_t n,
                              const unsigned char* __restrict__ pocket) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int s = seg[p];
        mask[p] = (s >= 0 && pocket[s]) ? 1 : 0;
    }
}

// Host: weighted union-find over the links; pocket[s] = 1 unless s's
// component has a link that contradicts the unit-cell offsets.
static int classify_segments(int n_seg, const std::vector<unsigned long long>& links,
                             std::vector<unsigned char>& pocket) {
    std::vector<int> parent(n_seg);
    std::vector<int> ox(n_seg, 0), oy(n_seg, 0), oz(n_seg, 0);  // offset to parent
    std::vector<unsigned char> bad(n_seg, 0);
    for (int s = 0; s < n_seg; ++s) parent[s] = s;
    auto find = [&](int s, int& x, int& y, int& z) {
        // returns the root and the offset of s relative to it; compresses
        int r = s;
        x = y = z = 0;
        while (parent[r] != r) {
            x += ox[r]; y += oy[r]; z += oz[r];
            r = parent[r];
        }
        int c = s, cx = x, cy = y, cz = z;
        while (parent[c] != c) {
            const int nxt = parent[c];
            const int tx = ox[c], ty = oy[c], tz = oz[c];
            parent[c] = r; ox[c] = cx; oy[c] = cy; oz[c] = cz;
            cx -= tx; cy -= ty; cz -= tz;
            c = nxt;
        }
        return r;
    };
    for (unsigned long long key : links) {
        const int dir = (int)(key & 15ull);
        const int to = (int)((key >> 4) & ((1ull << 30) - 1));
        const int from = (int)(key >> 34);
        if (from >= n_seg || to >= n_seg || dir < 1 || dir > 3) return -1;
        // uc(to) - uc(from) = e_dir (src/pocketblocking.cc:62-83)
        const int ex = dir == 1, ey = dir == 2, ez = dir == 3;
        int fx, fy, fz, tx, ty, tz;
        const int rf = find(from, fx, fy, fz);
        const int rt = find(to, tx, ty, tz);
        if (rf == rt) {
            if (tx - fx != ex || ty - fy != ey || tz - fz != ez) bad[rf] = 1;
        } else {
            parent[rt] = rf;
            ox[rt] = fx + ex - tx;
            oy[rt] = fy + ey - ty;
            oz[rt] = fz + ez - tz;
            bad[rf] |= bad[rt];
        }
    }
    pocket.assign(n_seg, 0);
    int n_pockets = 0;
    for (int s = 0; s < n_seg; ++s) {
        int x, y, z;
        const int r = find(s, x, y, z);
        pocket[s] = bad[r] ? 0 : 1;
        n_pockets += pocket[s];
    }
    return n_pockets;
}

// Steps 2-6 on a labelled grid (ps.lab), on stream st; fills ps.seg (segment
// per point) and ps.flags (pocket flag per segment, device) and returns the
// pocket count.
static int segment_and_classify(er_ctx* ctx, PocketScratch& ps, cudaStream_t st, int nx, int ny,
                                int nz, int* n_pockets) {
    const int64_t n = (int64_t)nx * ny * nz;
    int* lab = (int*)ps.lab.ptr;
    int* seg = (int*)ps.seg.ptr;
    const int gb = std::max(1, std::min<int>((int)((n + 255) / 256), ctx->num_sms * 16));
    {
        const int64_t tiles = (int64_t)((nz + kTK - 1) / kTK) * ((ny + kTJ - 1) / kTJ) *
                              ((nx + kTI - 1) / kTI);
        if (tiles > INT32_MAX) return set_error(ctx, ER_ERR_LIMIT, "pockets: grid too large");
        cc_union_tiles<<<(unsigned)tiles, 256, 0, st>>>(lab, nx, ny, nz);
        cc_union_faces<<<gb, 256, 0, st>>>(lab, nx, ny, nz);
    }
    cc_compress<<<gb, 256, 0, st>>>(lab, n);
    const int nblk = (int)((n + kScanItems - 1) / kScanItems);
    // p_misc: block counts (nblk) | block offsets (nblk + 1) | link count | table | list
    int* bcount = (int*)ps.misc.ptr;
    int* boff = bcount + nblk;
    int* nlink = boff + nblk + 1;
    cc_root_counts<<<nblk, 1024, 0, st>>>(lab, n, bcount);
    cc_scan_small<<<1, 1024, 0, st>>>(bcount, boff, nblk);
    int* rank = (int*)ps.grid.ptr;  // reuse: ranks live only until cc_segments
    cc_root_ranks<<<nblk, 1024, 0, st>>>(lab, n, boff, rank);
    cc_segments<<<gb, 256, 0, st>>>(lab, rank, n, seg);
    ER_CUDA(ctx, cudaGetLastError());
    int n_seg = 0;
    ER_CUDA(ctx, cudaMemcpyAsync(&n_seg, boff + nblk, sizeof(int), cudaMemcpyDeviceToHost, st));
    // face links
    const int64_t faces = (int64_t)ny * nz + (int64_t)nx * nz + (int64_t)nx * ny;
    int64_t tsize = 1024;
    while (tsize < 2 * faces) tsize <<= 1;
    const size_t misc_ints = (size_t)(2 * nblk + 2);
    const size_t tab_off = ((misc_ints * sizeof(int) + 255) / 256) * 256;
    unsigned long long* table = (unsigned long long*)((char*)ps.misc.ptr + tab_off);
    unsigned long long* list = table + tsize;
    ER_CUDA(ctx, cudaMemsetAsync(table, 0xff, tsize * sizeof(unsigned long long), st));
    ER_CUDA(ctx, cudaMemsetAsync(nlink, 0, sizeof(int), st));
    const int fb = std::max(1, std::min<int>((int)((faces + 255) / 256), ctx->num_sms * 8));
    cc_face_links<<<fb, 256, 0, st>>>(seg, nx, ny, nz, table, (int)(tsize - 1), list, nlink,
                                      (int)faces);
    ER_CUDA(ctx, cudaGetLastError());
    int nl = 0;
    ER_CUDA(ctx, cudaMemcpyAsync(&nl, nlink, sizeof(int), cudaMemcpyDeviceToHost, st));
    ER_CUDA(ctx, cudaStreamSynchronize(st));
    std::vector<unsigned long long> links(nl);
    if (nl) {
        ER_CUDA(ctx, cudaMemcpyAsync(links.data(), list, nl * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, st));
        ER_CUDA(ctx, cudaStreamSynchronize(st));
    }
    // a fixed order makes the host pass independent of the insertion order
    std::sort(links.begin(), links.end());
    std::vector<unsigned char> pocket;
    const int np = classify_segments(n_seg, links, pocket);
    if (np < 0) return set_error(ctx, ER_ERR_INVALID, "pockets: malformed face link");
    if (ps.flags.ensure_on(std::max<size_t>(pocket.size(), 1), ctx->pool, st) != ER_OK)
        return set_error(ctx, ER_ERR_NOMEM, "pockets: flag allocation");
    if (!pocket.empty()) {
        ER_CUDA(ctx, cudaMemcpyAsync(ps.flags.ptr, pocket.data(), pocket.size(),
                                     cudaMemcpyHostToDevice, st));
        ER_CUDA(ctx, cudaStreamSynchronize(st));  // `pocket` is freed on return
    }
    *n_pockets = np;
    return ER_OK;
}

static int ensure_pocket_scratch(er_ctx* ctx, PocketScratch& ps, cudaStream_t st, int nx, int ny,
                                 int nz, size_t grid_bytes) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t faces = (int64_t)ny * nz + (int64_t)nx * nz + (int64_t)nx * ny;
    int64_t tsize = 1024;
    while (tsize < 2 * faces) tsize <<= 1;
    const int nblk = (int)((n + kScanItems - 1) / kScanItems);
    const size_t misc_ints = (size_t)(2 * nblk + 2);
    const size_t tab_off = ((misc_ints * sizeof(int) + 255) / 256) * 256;
    const size_t misc = tab_off + (size_t)(tsize + faces) * sizeof(unsigned long long);
    cudaMemPool_t pool = ctx->pool;
    if (ps.lab.ensure_on(n * sizeof(int), pool, st) || ps.seg.ensure_on(n * sizeof(int), pool, st) ||
        ps.grid.ensure_on(std::max<size_t>(grid_bytes, n * sizeof(int)), pool, st) ||
        ps.misc.ensure_on(misc, pool, st))
        return set_error(ctx, ER_ERR_NOMEM, "pockets: device scratch allocation failed");
    return ER_OK;
}

static int check_dims(er_ctx* ctx, int nx, int ny, int nz, double T) {
    if (nx < 2 || ny < 2 || nz < 2) return set_error(ctx, ER_ERR_INVALID, "pockets: dims >= 2");
    if ((int64_t)nx * ny * nz >= (int64_t)INT32_MAX)
        return set_error(ctx, ER_ERR_LIMIT, "pockets: grid must have < 2^31 points");
    if (!std::isfinite(T)) return set_error(ctx, ER_ERR_INVALID, "pockets: temperature");
    return ER_OK;
}

}  // namespace er

using namespace er;

extern "C" int er_block_pockets(er_ctx* ctx, double* grid, int nx, int ny, int nz,
                                double temperature, int* n_pockets, int* segments_out) {
    er::NvtxRange nvtx("er_block_pockets");
    if (!ctx || !grid || !n_pockets) return ER_ERR_INVALID;
    int stt = check_dims(ctx, nx, ny, nz, temperature);
    if (stt != ER_OK) return stt;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    const int64_t n = (int64_t)nx * ny * nz;
    PocketScratch& ps = ctx->pocket;
    cudaStream_t st = ctx->stream;
    if ((stt = ensure_pocket_scratch(ctx, ps, st, nx, ny, nz, n * sizeof(double))) != ER_OK)
        return stt;
    if (ps.mask.ensure_on(n * sizeof(double), ctx->pool, st) != ER_OK)
        return set_error(ctx, ER_ERR_NOMEM, "pockets: grid allocation failed");
    double* dE = (double*)ps.mask.ptr;
    ER_CUDA(ctx, cudaMemcpyAsync(dE, grid, n * sizeof(double), cudaMemcpyHostToDevice, st));
    const int gb = std::max(1, std::min<int>((int)((n + 255) / 256), ctx->num_sms * 16));
    cc_init_f64<<<gb, 256, 0, st>>>(dE, n, 15.0 * temperature, (int*)ps.lab.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    int np = 0;
    if ((stt = segment_and_classify(ctx, ps, st, nx, ny, nz, &np)) != ER_OK) return stt;
    cc_block_f64<<<gb, 256, 0, st>>>(dE, (const int*)ps.seg.ptr, n,
                                     (const unsigned char*)ps.flags.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    ER_CUDA(ctx, cudaMemcpyAsync(grid, dE, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (segments_out)
        ER_CUDA(ctx, cudaMemcpyAsync(segments_out, ps.seg.ptr, n * sizeof(int),
                                     cudaMemcpyDeviceToHost, st));
    ER_CUDA(ctx, cudaStreamSynchronize(st));
    *n_pockets = np;
    return ER_OK;
}

namespace er {

int block_pockets_device_on(er_ctx* ctx, PocketScratch& ps, cudaStream_t st, const float* grid,
                            int nx, int ny, int nz, double temperature, uint8_t* mask_out,
                            int* n_pockets) {
    int stt = check_dims(ctx, nx, ny, nz, temperature);
    if (stt != ER_OK) return stt;
    const int64_t n = (int64_t)nx * ny * nz;
    if ((stt = ensure_pocket_scratch(ctx, ps, st, nx, ny, nz, 0)) != ER_OK) return stt;
    const int gb = std::max(1, std::min<int>((int)((n + 255) / 256), ctx->num_sms * 16));
    cc_init_f32<<<gb, 256, 0, st>>>(grid, n, 15.0 * temperature, (int*)ps.lab.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    int np = 0;
    if ((stt = segment_and_classify(ctx, ps, st, nx, ny, nz, &np)) != ER_OK) return stt;
    cc_block_mask<<<gb, 256, 0, st>>>(mask_out, (const int*)ps.seg.ptr, n,
                                      (const unsigned char*)ps.flags.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    ER_CUDA(ctx, cudaStreamSynchronize(st));
    *n_pockets = np;
    return ER_OK;
}

}  // namespace er

extern "C" int er_block_pockets_device(er_ctx* ctx, const float* grid, int nx, int ny, int nz,
                                       double temperature, uint8_t* pocket_mask_out,
                                       int* n_pockets) {
    er::NvtxRange nvtx("er_block_pockets_device");
    if (!ctx || !grid || !pocket_mask_out || !n_pockets) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    return block_pockets_device_on(ctx, ctx->pocket, ctx->stream, grid, nx, ny, nz, temperature,
                                   pocket_mask_out, n_pockets);
}

// ------------------------------------------------------------------ accessibility
// ComputeGridSheetAccessibleOrNot (src/computegridsheet.h:101-165): a point is
// inaccessible (0) when some atom image within +-1 cells has r^2 < sigma_mix^2.
// Image positions and r^2 follow the reference's FP64 expressions without
// contraction, so the mask is bit-exact.
namespace er {

struct AccParams {
    double t[9];
    int nx, ny, nz;
};

__device__ __forceinline__ void acc_cart(const double* t, double xf, double yf, double zf,
                                         double& x, double& y, double& z) {
    x = __dadd_rn(__dadd_rn(__dmul_rn(t[0], xf), __dmul_rn(t[1], yf)), __dmul_rn(t[2], zf));
    y = __dadd_rn(__dadd_rn(__dmul_rn(t[3], xf), __dmul_rn(t[4], yf)), __dmul_rn(t[5], zf));
    z = __dadd_rn(__dadd_rn(__dmul_rn(t[6], xf), __dmul_rn(t[7], yf)), __dmul_rn(t[8], zf));
}

__global__ void acc_images_kernel(const double4* __restrict__ atoms, int n, AccParams P,
                                  double4* __restrict__ img) {
    const int total = 27 * n;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        const int a = q / 27, m = q % 27;
        const int i = m / 9 - 1, j = (m / 3) % 3 - 1, k = m % 3 - 1;
        const double4 at = atoms[a];
        double x, y, z;
        // src/computegridsheet.h:134-140
        acc_cart(P.t, __dadd_rn(at.x, (double)i), __dadd_rn(at.y, (double)j),
                 __dadd_rn(at.z, (double)k), x, y, z);
        img[q] = make_double4(x, y, z, at.w);
    }
}

__global__ void __launch_bounds__(256) acc_grid_kernel(const double4* __restrict__ img, int nimg,
                                                       AccParams P, uint8_t* __restrict__ out) {
    __shared__ double4 tile[512];
    const int64_t n = (int64_t)P.nx * P.ny * P.nz;
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double x = 0, y = 0, z = 0;
    bool live = p < n, overlap = false;
    if (live) {
        const int k = (int)(p % P.nz), j = (int)((p / P.nz) % P.ny),
                  i = (int)(p / ((int64_t)P.ny * P.nz));
        acc_cart(P.t, __ddiv_rn((double)i, (double)(P.nx - 1)),
                 __ddiv_rn((double)j, (double)(P.ny - 1)),
                 __ddiv_rn((double)k, (double)(P.nz - 1)), x, y, z);
    }
    for (int base = 0; base < nimg; base += 512) {
        const int cnt = min(512, nimg - base);
        __syncthreads();
        for (int q = threadIdx.x; q < cnt; q += blockDim.x) tile[q] = img[base + q];
        __syncthreads();
        if (live && !overlap) {
            for (int q = 0; q < cnt; ++q) {
                const double4 w = tile[q];
                const double dx = __dsub_rn(x, w.x), dy = __dsub_rn(y, w.y),
                             dz = __dsub_rn(z, w.z);
                const double r2 =
                    __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                if (r2 < w.w) {  // src/computegridsheet.h:148
                    overlap = true;
                    break;
                }
            }
        }
    }
    if (live) out[p] = overlap ? 0 : 1;
}

}  // namespace er

extern "C" int er_accessibility(er_ctx* ctx, int fw_id, int nx, int ny, int nz, uint8_t* out) {
    if (!ctx || !out) return ER_ERR_INVALID;
    if (int st = er::check_grid_dims(ctx, nx, ny, nz, "accessibility")) return st;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    const er::FwRecord* f = er::find_fw(ctx, fw_id);
    if (!f) return er::set_error(ctx, ER_ERR_NOT_FOUND, "accessibility: unknown framework id");
    const int64_t n = (int64_t)nx * ny * nz;
    const int nimg = 27 * f->n_atoms;
    if (ctx->pocket.lab.ensure(std::max<size_t>((size_t)nimg, 1) * sizeof(double4)) ||
        ctx->pocket.seg.ensure((size_t)n))
        return er::set_error(ctx, ER_ERR_NOMEM, "accessibility: scratch allocation failed");
    er::AccParams P;
    for (int k = 0; k < 9; ++k) P.t[k] = f->t[k];
    P.nx = nx; P.ny = ny; P.nz = nz;
    cudaStream_t st = ctx->stream;
    double4* img = (double4*)ctx->pocket.lab.ptr;
    if (nimg > 0)
        er::acc_images_kernel<<<std::max(1, std::min((nimg + 255) / 256, ctx->num_sms * 8)), 256,
                                0, st>>>(f->dev.atom_frac, f->n_atoms, P, img);
    er::acc_grid_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(img, nimg, P,
                                                                     (uint8_t*)ctx->pocket.seg.ptr);
    ER_CUDA(ctx, cudaGetLastError());
    ER_CUDA(ctx, cudaMemcpyAsync(out, ctx->pocket.seg.ptr, (size_t)n, cudaMemcpyDeviceToHost, st));
    ER_CUDA(ctx, cudaStreamSynchronize(st));
    return ER_OK;
}
