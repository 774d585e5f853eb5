// er_engine.cuh -- the probe-framework Lennard-Jones pair-sum engine (sm_100a).
//
// What it computes is the sum of src/computegridsheet.h:54-92 (and the same
// sum in src/doHenry.h:70-98): at every point p, over every kept atom image
// a + T n, 4 eps s^6 (s^6 - 1) with s = sig^2 / r^2 when r^2 < rc^2.
// How it computes it is its own:
//
//  * Positions live in the framework's positioning frame R (an upper-
//    triangular rotation of the cell matrix T, equal to T bit for bit when T
//    is already upper triangular, as the reference's cells are). Distances are
//    frame-independent; the exact cutoff decision below still uses T.
//  * A CTA owns up to 8 warp tasks of <= 32*P points (a lattice sub-brick of
//    the grid, or a chunk of one spatial bin of Widom insertions). The CTA box
//    is the FP64 bounding box of its points; all FP32 coordinates are relative
//    to the box centre, so FP32 never holds magnitudes above rc + box.
//  * Candidate atom images come from the framework's cell list: one contiguous
//    image range per (y, z) row of cells, with the x range of each row pruned
//    by the cutoff circle. Passing candidates are compacted in order (block
//    scans, so the order is deterministic) into shared memory.
//  * Each warp splits the CTA candidates against its own box into an inner
//    list (inside the cutoff for every point of the warp: no test needed) and
//    a shell list (cutoff tested per pair). Lists are u16 byte offsets.
//  * Lattice points of one lane differ only along the grid's first axis, which
//    R maps to Cartesian x; so per atom the lane forms dy^2 + dz^2 once and per
//    point only dx and r^2 = dx^2 + (dy^2 + dz^2). Point pairs run as packed
//    FP32x2 instructions (add/mul/fma .f32x2): per two pair terms 5 packed ops
//    and 2 MUFU.RCP, E += u^3 (C12 u^3 - C6), u = 1 / r^2.
//  * Shell pairs whose FP32 r^2 lies within a proven error window of rc^2 are
//    re-decided in FP64 with the reference's own expression order, so the set
//    of summed pairs equals the FP64 reference's set exactly.
//  * Accumulation: FP32 over chunks of 64 atoms, chunk sums added into FP64
//    per-point totals (ER_PREC_COMP, ER_PREC_NEAR64), or FP32 over the whole
//    list (ER_PREC_FP32). ER_PREC_NEAR64 (the default) evaluates the pairs of
//    atoms within kNearR of a warp's points in FP64: those large terms carry
//    the FP32 error where they cancel to a small |E|.
#pragma once
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "er_internal.h"
#include "er_philox.h"

namespace er {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
// points per thread (P) and the CTA brick are set by the point policy (Tile)
constexpr int kWJ = 4, kWK = 8;            // lanes of a warp sub-brick along j, k
constexpr int kPMax = 8;                   // largest P any policy uses
constexpr int kMaxCand = 1024;             // CTA candidate capacity per flush
constexpr int kRowChunk = kThreads;        // cell rows examined per producer pass
constexpr int kAccChunk = 64;              // atoms per FP32 partial sum (shell lists,
                                           // and every list of ER_PREC_COMP)
constexpr float kEnergyCap = 1.0e30f;      // overflow cap (ER_ENERGY_CAP)

// PREC_COUNT writes the number of in-cutoff pair terms per point instead of
// the energy (same traversal; used to count the algorithmic work of a job).
// PREC_NEAR64 is PREC_COMP with the pairs of atoms within kNearR of a warp's
// box evaluated in FP64 (they carry most of |E| where terms cancel).
// PREC_FP64 evaluates every pair term in FP64 (same pair set).
enum { PREC_COMP = 0, PREC_FP32 = 1, PREC_COUNT = 2, PREC_NEAR64 = 3, PREC_FP64 = 4 };

template <int PREC>
struct PrecTraits {
    static constexpr bool comp = PREC == PREC_COMP || PREC == PREC_NEAR64;
    static constexpr bool near64 = PREC == PREC_NEAR64;
    static constexpr bool fp64 = PREC == PREC_FP64;
    // Atoms per FP32 partial sum of an inner list. Once NEAR64 has taken the
    // near terms to FP64, the rounding of the FP32 partial sums (its error
    // grows with the chunk length times the partial's magnitude) is what is
    // left: 16-atom partials keep every E < -10 K point of the 256-framework
    // batch within 1e-5 of FP64, 64-atom ones leave 82 of 1.4e8 above it;
    // 32-atom ones were 0.8 % faster but raised the sampled p99 error from
    // 5.1e-7 to 6.6e-7.
    static constexpr int inner_chunk = PREC == PREC_NEAR64 ? 16 : 64;
};

constexpr int kNearCap = 256;     // near-list capacity per warp (overflow stays FP32)
constexpr int kRec = 3;           // borderline shell atoms recorded per thread and flush
                                  // (10-bit list positions packed in one register)
constexpr float kNearR = 5.0f;    // near radius (A) from the warp box

// One candidate atom image in shared memory (32 bytes, so a list entry can be
// the byte offset of its record). x, C12 and -C6 are stored twice so that a
// 128-bit load yields them as packed FP32x2 operands; the position is the
// first 16 bytes (one vector load in the per-warp split).
struct __align__(32) Cand {
    float ax, ax_, ay, az;       // x (twice), y, z relative to the CTA centre
    float c12, c12_, nc6, nc6_;  // C12 (twice), -C6 (twice)
};

struct __align__(32) EngineSmem {
    Cand cand[kMaxCand];                   // CTA candidates
    int cid[kMaxCand];                     // their image indices (FP64 paths)
    unsigned short wl[kWarps][kMaxCand];   // per-warp inner (front) / shell (back) lists of
                                           // byte offsets into cand
    unsigned short wn[kWarps][kNearCap];   // per-warp near lists (PREC_NEAR64): atoms inside
                                           // the cutoff for every point (front) and atoms
                                           // crossing it (back)
    double tot[kPMax][kThreads];           // FP64 per-point sums, [p][thread]
    int row_beg[kRowChunk];
    int row_off[kRowChunk];
    int warp_tot[kWarps];
    double red[kWarps][6];
    double box[6];                         // CTA box (FP64 lo, hi)
    float wbox[kWarps][6];                 // warp boxes (local FP32 lo, hi)
    int item, task;                        // persistent-queue item and its task
    unsigned long long mbar[2];            // completion barriers of the staged cell rows
};

// ----------------------------------------------------------- packed FP32x2
typedef unsigned long long f2_t;

__device__ __forceinline__ f2_t f2_pack(float lo, float hi) {
    f2_t d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ void f2_unpack(f2_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b) {
    f2_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
    f2_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
    f2_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
    f2_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// 1.0f when a < b, else 0.0f
__device__ __forceinline__ float set_lt(float a, float b) {
    float d;
    asm("set.lt.f32.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ------------------------------------------------ bulk copies (TMA engine)
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// the single arrival of a phase, announcing the bytes the phase's copies bring
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// Waits for the phase of `parity` to complete; false after kMbarSpins polls
// (a copy that never lands: the caller records the fault instead of hanging).
constexpr int kMbarSpins = 1 << 22;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity,
                                          int spins = kMbarSpins) {
    const unsigned a = smem_u32(bar);
    for (int i = 0; i < spins; ++i) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// global -> shared copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) by the bulk-copy engine, completing on `bar`; one CTA, no multicast
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Exclusive block scan of one int per thread; *total gets the block sum.
__device__ __forceinline__ int block_exscan(int v, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < kWarps ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kWarps) warp_tot[lane] = t;
    }
    __syncthreads();
    int base = w ? warp_tot[w - 1] : 0;
    *total = warp_tot[kWarps - 1];
    __syncthreads();
    return base + x - v;
}

__device__ __forceinline__ void frac_to_cart(const double* t, double xf, double yf, double zf,
                                             double& x, double& y, double& z) {
    // src/computegridsheet.h:25-27, strict IEEE order (no contraction)
    x = __dadd_rn(__dadd_rn(__dmul_rn(t[0], xf), __dmul_rn(t[1], yf)), __dmul_rn(t[2], zf));
    y = __dadd_rn(__dadd_rn(__dmul_rn(t[3], xf), __dmul_rn(t[4], yf)), __dmul_rn(t[5], zf));
    z = __dadd_rn(__dadd_rn(__dmul_rn(t[6], xf), __dmul_rn(t[7], yf)), __dmul_rn(t[8], zf));
}

// The reference's FP64 in-cutoff decision for point f and image gid:
// src/computegridsheet.h:61-79 evaluated in IEEE double without contraction,
// in the caller's cell matrix T.
static __device__ __noinline__ bool exact_in_cutoff(const FwDev& fw, const double* f, int gid,
                                                    double r2min) {
    const uint32_t id = fw.img_id[gid];
    const int atom = (int)(id / (uint32_t)fw.imgs_per_atom);
    const int m = (int)(id - (uint32_t)atom * (uint32_t)fw.imgs_per_atom);
    const int n2 = 2 * fw.rep[2] + 1, n1 = 2 * fw.rep[1] + 1;
    const int kk = m % n2 - fw.rep[2];
    const int jj = (m / n2) % n1 - fw.rep[1];
    const int ii = m / (n2 * n1) - fw.rep[0];
    const double4 a = fw.atom_frac[atom];
    double x, y, z, xw, yw, zw;
    frac_to_cart(fw.t, f[0], f[1], f[2], x, y, z);
    frac_to_cart(fw.t, __dadd_rn(a.x, (double)ii), __dadd_rn(a.y, (double)jj),
                 __dadd_rn(a.z, (double)kk), xw, yw, zw);
    const double dx = __dsub_rn(x, xw), dy = __dsub_rn(y, yw), dz = __dsub_rn(z, zw);
    double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    r2 = (r2 > r2min) ? r2 : r2min;
    return r2 < fw.rc2;
}

// One atom image for FP64 pair terms: position relative to the CTA centre and
// FP64 (C12, C6).
struct Atom64 {
    double x, y, z, c12, c6;
};
__device__ __forceinline__ Atom64 atom64(const FwDev& fw, int gid, double o0, double o1,
                                         double o2) {
    const double4 a = fw.img_xyz[gid];
    const double2 lj = fw.img_lj64[gid];
    return Atom64{a.x - o0, a.y - o1, a.z - o2, lj.x, lj.y};
}
// FP64 pair term of atom a at a point q (both relative to the CTA centre),
// with the correctly rounded reciprocal (ER_PREC_FP64, the reference mode of
// the precision sweeps).
__device__ __forceinline__ double pair64(const Atom64& a, double qx, double qy, double qz,
                                         double r2min) {
    const double dx = qx - a.x, dy = qy - a.y, dz = qz - a.z;
    double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
    r2 = fmax(r2, r2min);
    const double u = __drcp_rn(r2);
    const double u3 = u * u * u;
    return u3 * fma(a.c12, u3, -a.c6);
}
// 1/x in FP64 for the near pairs of PREC_NEAR64: one Newton step
// y = y0 (1 + e), e = 1 - x y0, from the hardware seed y0 =
// rcp.approx.ftz.f64(x), whose relative error e0 is below 2^-16 (asserted by
// the tests; er_probe_rcp64_seed measures 9.9e-7, about 2^-20), leaves a
// relative error of order e0^2 < 2^-32 plus two FP64 roundings. A near term then carries at
// most ~6 x 2^-32 of its own size, far below the 1e-5 relative bound on the
// energy even where near terms cancel a thousandfold (a third-order step,
// e0^3, gave the same errors on 71,378 sampled E < -10 K points of the
// 256-framework batch and took 0.8 % longer; a seed from the FP32
// reciprocal, converted, took 4.7 % longer). x is a squared distance,
// clamped to >= min_r^2 > 0 by the caller, so the seed is finite and normal.
__device__ __forceinline__ double rcp64_nr(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
// acc + the FP64 pair term of a near pair (PREC_NEAR64): r^2 = dx^2 + yzc from
// dx and yzc = dy^2 + dz^2 + min_r^2, formed once per atom and lane, with the
// reference's clamp r^2 >= min_r^2 (src/computegridsheet.h:77) folded into
// yzc: both keep r^2 >= min_r^2, and min_r^2 (1e-24 or 1e-32 A^2) lies below
// the FP64 resolution of r^2 unless r^2 < ~1e-8 A^2, a point within 1e-4 A of
// an atom, whose energy (> 1e40 K) is capped either way. (The clamp as a
// separate FP64 max cost 3 % of the 256-framework batch.) Reciprocal by
// rcp64_nr, the term added by one FMA.
__device__ __forceinline__ double near_acc64(double acc, double dx, double yzc, double c12,
                                             double c6) {
    const double u = rcp64_nr(fma(dx, dx, yzc));
    const double u3 = u * u * u;
    return fma(u3, fma(c12, u3, -c6), acc);
}

// FP32 r^2 of the generic form (each point has its own x, y, z) and of the
// lattice form (ss = dy^2 + dz^2 shared by a lane's points). Both are fixed
// instruction sequences, so a later re-evaluation reproduces the same bits.
__device__ __forceinline__ float r2_generic(float px, float py, float pz, float ax, float ay,
                                            float az) {
    const float dx = __fsub_rn(px, ax);
    const float dy = __fsub_rn(py, ay);
    const float dz = __fsub_rn(pz, az);
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}
__device__ __forceinline__ float ss_lattice(float py, float pz, float ay, float az) {
    const float dy = __fsub_rn(py, ay);
    const float dz = __fsub_rn(pz, az);
    return __fmaf_rn(dz, dz, __fmul_rn(dy, dy));
}
__device__ __forceinline__ float r2_lattice(float px, float ax, float ss) {
    const float dx = __fsub_rn(px, ax);
    return __fmaf_rn(dx, dx, ss);
}
// E_pair = u3 * t with u = 1/r^2, u3 = u^3, t = C12 u3 - C6.
__device__ __forceinline__ float pair_term(float r2, float c12, float nc6) {
    const float u = rcp_approx(r2);
    const float u3 = __fmul_rn(__fmul_rn(u, u), u);
    return __fmul_rn(u3, __fmaf_rn(c12, u3, nc6));
}

// ---------------------------------------------------------------------------
// Point sources. A policy maps (warp, lane, p) to an FP64 fractional point
// and stores its energy. kLattice: a lane's P points differ only in the
// first fractional coordinate.

// Lattice points of one (2P) x 8 x 16 brick of a grid job: warp w owns the
// P x 4 x 8 sub-brick at ((w & 1) P, ((w >> 1) & 1) 4, (w >> 2) 8); lane l the
// (j, k) = (l / 8, l % 8) column of it and its P points along i.
template <int P_>
struct GridPolicy {
    static constexpr int kP = P_;
    static constexpr bool kLattice = true;
    static constexpr int kBI = 2 * P_, kBJ = 2 * kWJ, kBK = 2 * kWK;
    const GridTask* T;
    int i0, j0, k0;
    __device__ GridPolicy(const GridTask* task, int brick) : T(task) {
        const int nbk = task->nb[2], nbj = task->nb[1];
        const int bk = brick % nbk;
        const int bj = (brick / nbk) % nbj;
        const int bi = brick / (nbk * nbj);
        i0 = bi * kBI; j0 = bj * kBJ; k0 = bk * kBK;
    }
    __device__ __forceinline__ void index(int w, int lane, int p, int& i, int& j, int& k) const {
        i = i0 + (w & 1) * kP + p;
        j = j0 + ((w >> 1) & 1) * kWJ + lane / kWK;
        k = k0 + (w >> 2) * kWK + lane % kWK;
    }
    // Out-of-range points are clamped onto the lattice (same j, k when only i
    // overshoots, so a lane's points keep sharing y and z) and never stored.
    __device__ __forceinline__ bool point(int w, int lane, int p, double* f) const {
        int i, j, k;
        index(w, lane, p, i, j, k);
        const bool ok = i < T->nx && j < T->ny && k < T->nz;
        i = min(i, T->nx - 1); j = min(j, T->ny - 1); k = min(k, T->nz - 1);
        // axes 1.0 * i / (N - 1), src/writegrid.cu:122-127
        f[0] = __ddiv_rn((double)i, (double)(T->nx - 1));
        f[1] = __ddiv_rn((double)j, (double)(T->ny - 1));
        f[2] = __ddiv_rn((double)k, (double)(T->nz - 1));
        return ok;
    }
    // the point's Cartesian position in the positioning frame r
    __device__ __forceinline__ bool cart(const double* r, int w, int lane, int p, double& x,
                                         double& y, double& z) const {
        double f[3];
        const bool ok = point(w, lane, p, f);
        frac_to_cart(r, f[0], f[1], f[2], x, y, z);
        return ok;
    }
    __device__ __forceinline__ void store(int w, int lane, int p, float e) const {
        int i, j, k;
        index(w, lane, p, i, j, k);
        if (i < T->nx && j < T->ny && k < T->nz)
            // streaming store: the grid is written once and not read back here,
            // so its lines are the first the L2 evicts
            __stcs(&T->out[(size_t)k + (size_t)j * T->nz + (size_t)i * T->ny * T->nz], e);
    }
    __device__ __forceinline__ void store64(int w, int lane, int p, double e) const {
        int i, j, k;
        index(w, lane, p, i, j, k);
        if (i < T->nx && j < T->ny && k < T->nz)
            T->out64[(size_t)k + (size_t)j * T->nz + (size_t)i * T->ny * T->nz] = e;
    }
};

// Widom insertion points: CTA c owns sorted positions [256 P c, 256 P (c + 1))
// of `order` (points stored in that order); warp w the 32 P positions from
// 256 P c + 32 P w, lane l position p * 32 + l of them.
template <int P_>
struct PointPolicy {
    static constexpr int kP = P_;
    static constexpr bool kLattice = false;
    const PointTask* T;
    int base, nv;
    __device__ PointPolicy(const PointTask* task, int cta)
        : T(task), base(cta * kWarps * 32 * kP), nv(*task->n_valid) {}
    __device__ __forceinline__ int slot_index(int w, int lane, int p) const {
        const int pos = base + w * (32 * kP) + p * 32 + lane;
        return pos < nv ? T->order[pos] : -1;
    }
    __device__ __forceinline__ int pos_of(int w, int lane, int p, bool& ok) const {
        const int pos = base + w * (32 * kP) + p * 32 + lane;
        ok = pos < nv;
        return ok ? pos : min(base, nv - 1);  // a finite stand-in, never stored
    }
    // Cartesian position (frame r), stored at its bin-order position by the
    // placement pass
    __device__ __forceinline__ bool cart(const double*, int w, int lane, int p, double& x,
                                         double& y, double& z) const {
        bool ok;
        const int pos = pos_of(w, lane, p, ok);
        x = T->pts[3 * (size_t)pos];
        y = T->pts[3 * (size_t)pos + 1];
        z = T->pts[3 * (size_t)pos + 2];
        return ok;
    }
    // fractional position, regenerated from the insertion's Philox counter
    // (only the exact cutoff decisions need it)
    __device__ __forceinline__ bool point(int w, int lane, int p, double* f) const {
        bool ok;
        const int pos = pos_of(w, lane, p, ok);
        insertion_point(T->seed, (uint64_t)T->order[pos], f);
        return ok;
    }
    __device__ __forceinline__ void store(int w, int lane, int p, float e) const {
        const int idx = slot_index(w, lane, p);
        if (idx >= 0) T->energies[idx] = e;
    }
    __device__ __forceinline__ void store64(int w, int lane, int p, double e) const {
        store(w, lane, p, (float)e);
    }
};

// ---------------------------------------------------------------------------
// Half-width (in ulps of fl32(rc^2)) of the window around rc^2 inside which
// an FP32 r^2 may sit on the other side of rc^2 from the exact FP64 r^2.
// Coordinates relative to the CTA centre are bounded by M = rc + margin +
// box diagonal; each displacement component then carries at most 1.5 ulp(M)
// of rounding (two roundings into FP32, one subtraction), which moves r^2 by
// at most 2 sqrt(3) rc * 1.5 ulp(M) near the cutoff; the FMUL/FFMA chain adds
// at most 1.5 ulp(rc^2). The window is twice that bound plus two ulps.
__device__ __forceinline__ int borderline_ulps(double rc, float rc2f, double box_diag) {
    const double M = rc + 1e-3 + box_diag;
    int e;
    frexp(M, &e);
    const double ulpM = ldexp(1.0, e - 24);
    frexp((double)rc2f, &e);
    const double ulpR = ldexp(1.0, e - 24);
    const double err = 2.0 * 1.7320508075688772 * rc * 1.5 * ulpM + 1.5 * ulpR + 1e-9;
    return 2 * ((int)ceil(err / ulpR) + 2);
}

// Per-thread state of one CTA pass. The FP64 per-point sums live in shared
// memory (EngineSmem::tot), the warp box and the CTA centre too.
template <class Pol, int PREC>
struct Lane {
    static constexpr int P = Pol::kP;
    static constexpr int NY = Pol::kLattice ? 1 : P;  // distinct y, z per lane
    float px[P], py[NY], pz[NY];
    unsigned vmask;
    bool warp_live;
    int bul;
};

__device__ __forceinline__ double& tot_at(EngineSmem& s, int p) {
    return s.tot[p][threadIdx.x];
}

// Folds FP32 chunk sums into FP64 registers.
template <int M>
__device__ __forceinline__ void fold_regs(double* acc64, f2_t* acc2) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float a0, a1;
        f2_unpack(acc2[m], a0, a1);
        acc64[2 * m] += (double)a0;
        acc64[2 * m + 1] += (double)a1;
        acc2[m] = 0ull;
    }
}

// Folds FP32 chunk sums into the FP64 totals.
template <int M>
__device__ __forceinline__ void fold_packed(EngineSmem& s, f2_t* acc2) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
        float a0, a1;
        f2_unpack(acc2[m], a0, a1);
        tot_at(s, 2 * m) += (double)a0;
        tot_at(s, 2 * m + 1) += (double)a1;
        acc2[m] = 0ull;
    }
}

__device__ __forceinline__ void cta_centre(const EngineSmem& s, double& o0, double& o1,
                                           double& o2) {
    o0 = 0.5 * (s.box[0] + s.box[3]);
    o1 = 0.5 * (s.box[1] + s.box[4]);
    o2 = 0.5 * (s.box[2] + s.box[5]);
}

// Lattice inner list: every pair inside the cutoff, packed over point pairs.
template <class Pol, int PREC>
__device__ __forceinline__ void lattice_inner(EngineSmem& s, const unsigned short* wl,
                                              int n_in, Lane<Pol, PREC>& L) {
    constexpr int M = Pol::kP / 2;
    constexpr bool kComp = PrecTraits<PREC>::comp;
    constexpr int kChunk = PrecTraits<PREC>::inner_chunk;
    f2_t px2[M], acc2[M];
    double acc64[2 * M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        px2[m] = f2_pack(L.px[2 * m], L.px[2 * m + 1]);
        acc2[m] = 0ull;
        acc64[2 * m] = acc64[2 * m + 1] = 0.0;
    }
    const f2_t one2 = f2_pack(1.0f, 1.0f);
    const float py = L.py[0], pz = L.pz[0];
    const char* cbase = reinterpret_cast<const char*>(s.cand);
    const unsigned* wl32 = reinterpret_cast<const unsigned*>(wl);
    auto atom = [&](unsigned off) {
        const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(cbase + off);       // x x | y z
        const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(cbase + off + 16);  // C12 | -C6
        if (PREC == PREC_COUNT) {
#pragma unroll
            for (int m = 0; m < M; ++m) acc2[m] = f2_add(acc2[m], one2);
            return;
        }
        float ay, az;
        f2_unpack(v0.y, ay, az);
        const float ss = ss_lattice(py, pz, ay, az);
        const f2_t ss2 = f2_pack(ss, ss);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const f2_t dx = f2_sub(px2[m], v0.x);
            const f2_t r2 = f2_fma(dx, dx, ss2);
            float r0, r1;
            f2_unpack(r2, r0, r1);
            const f2_t u = f2_pack(rcp_approx(r0), rcp_approx(r1));
            const f2_t u3 = f2_mul(f2_mul(u, u), u);
            acc2[m] = f2_fma(u3, f2_fma(v1.x, u3, v1.y), acc2[m]);
        }
    };
    int q = 0;
    while (q < n_in) {
        const int qe = kComp ? min(q + kChunk, n_in) : n_in;
        // eight atoms per iteration (one 128-bit load of their list entries):
        // more independent chains between the MUFU results (256-framework
        // batch: 350 -> 342 ms against two atoms per iteration)
        for (; q + 7 < qe; q += 8) {  // q is a multiple of 8 here (chunk starts are)
            const uint4 eight = *reinterpret_cast<const uint4*>(wl32 + (q >> 1));
            atom(eight.x & 0xffffu);
            atom(eight.x >> 16);
            atom(eight.y & 0xffffu);
            atom(eight.y >> 16);
            atom(eight.z & 0xffffu);
            atom(eight.z >> 16);
            atom(eight.w & 0xffffu);
            atom(eight.w >> 16);
        }
        for (; q + 3 < qe; q += 4) {
            const uint2 four = *reinterpret_cast<const uint2*>(wl32 + (q >> 1));
            atom(four.x & 0xffffu);
            atom(four.x >> 16);
            atom(four.y & 0xffffu);
            atom(four.y >> 16);
        }
        for (; q + 1 < qe; q += 2) {  // q is even here: chunks have an even length
            const unsigned two = wl32[q >> 1];
            atom(two & 0xffffu);
            atom(two >> 16);
        }
        if (q < qe) atom(wl[q++]);
        fold_regs<M>(acc64, acc2);
    }
#pragma unroll
    for (int p = 0; p < 2 * M; ++p) tot_at(s, p) += acc64[p];
}

// Lattice shell list: cutoff tested per pair (mask 1.0 / 0.0), and the
// smallest |r^2 - fl32(rc^2)| per point pair kept for the borderline test.
template <class Pol, int PREC>
__device__ __forceinline__ int lattice_shell(EngineSmem& s, const unsigned short* wl, int n_sh,
                                             float rc2f, float win, Lane<Pol, PREC>& L,
                                             unsigned& rec) {
    constexpr int M = Pol::kP / 2;
    constexpr bool kComp = PrecTraits<PREC>::comp;
    f2_t px2[M], acc2[M];
    int nrec = 0;
    rec = 0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
        px2[m] = f2_pack(L.px[2 * m], L.px[2 * m + 1]);
        acc2[m] = 0ull;
    }
    const f2_t rc2 = f2_pack(rc2f, rc2f);
    const float py = L.py[0], pz = L.pz[0];
    const char* cbase = reinterpret_cast<const char*>(s.cand);
    // the shell list runs backwards from the end of wl
    const unsigned* wl32 = reinterpret_cast<const unsigned*>(wl);
    auto atom = [&](unsigned off, int q) {
        const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(cbase + off);       // x x | y z
        const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(cbase + off + 16);  // C12 | -C6
        float ay, az;
        f2_unpack(v0.y, ay, az);
        const float ss = ss_lattice(py, pz, ay, az);
        const f2_t ss2 = f2_pack(ss, ss);
        float mn = INFINITY;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const f2_t dx = f2_sub(px2[m], v0.x);
            const f2_t r2 = f2_fma(dx, dx, ss2);
            float r0, r1, d0, d1;
            f2_unpack(r2, r0, r1);
            const f2_t in = f2_pack(set_lt(r0, rc2f), set_lt(r1, rc2f));
            f2_unpack(f2_sub(r2, rc2), d0, d1);
            mn = fminf(mn, fminf(fabsf(d0), fabsf(d1)));
            if (PREC == PREC_COUNT) {
                acc2[m] = f2_add(acc2[m], in);
            } else {
                const f2_t u = f2_pack(rcp_approx(r0), rcp_approx(r1));
                const f2_t u3 = f2_mul(f2_mul(u, u), u);
                acc2[m] = f2_fma(f2_mul(u3, in), f2_fma(v1.x, u3, v1.y), acc2[m]);
            }
        }
        if (mn <= win) {  // rare: a pair of this atom sits near the cutoff
            rec = (rec << 10) | (unsigned)q;
            ++nrec;
        }
    };
    int q = 0;
    while (q < n_sh) {
        const int qe = kComp ? min(q + kAccChunk, n_sh) : n_sh;
        for (; q + 1 < qe; q += 2) {
            // entries q, q+1 sit at wl[K-1-q], wl[K-2-q]: one aligned u32
            const unsigned two = wl32[(kMaxCand - 2 - q) >> 1];
            atom(two >> 16, q);
            atom(two & 0xffffu, q + 1);
        }
        if (q < qe) {
            atom(wl[kMaxCand - 1 - q], q);
            ++q;
        }
        if (kComp) fold_packed<M>(s, acc2);
    }
    if (!kComp) fold_packed<M>(s, acc2);
    return nrec;
}

// Generic (per-point x, y, z) inner and shell lists, packed over point pairs
// (2m, 2m + 1): per two pair terms 9 packed FP32x2 instructions and 2
// MUFU.RCP; r^2 = fma(dz, dz, fma(dy, dy, dx * dx)) as in r2_generic, so the
// borderline re-check reproduces it bit for bit.
template <class Pol, int PREC>
__device__ __forceinline__ int generic_packed_lists(EngineSmem& s, const unsigned short* wl,
                                                    int n_in, int n_sh, float rc2f, float win,
                                                    Lane<Pol, PREC>& L, unsigned& rec) {
    constexpr int M = Pol::kP / 2;
    constexpr bool kComp = PrecTraits<PREC>::comp;
    f2_t px2[M], py2[M], pz2[M], acc2[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
        px2[m] = f2_pack(L.px[2 * m], L.px[2 * m + 1]);
        py2[m] = f2_pack(L.py[2 * m], L.py[2 * m + 1]);
        pz2[m] = f2_pack(L.pz[2 * m], L.pz[2 * m + 1]);
        acc2[m] = 0ull;
    }
    const f2_t one2 = f2_pack(1.0f, 1.0f);
    const f2_t rc2 = f2_pack(rc2f, rc2f);
    const char* cbase = reinterpret_cast<const char*>(s.cand);
    int nrec = 0;
    rec = 0;
    auto inner_atom = [&](unsigned off) {
        const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(cbase + off);       // x x | y z
        const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(cbase + off + 16);  // C12 | -C6
        if (PREC == PREC_COUNT) {
#pragma unroll
            for (int m = 0; m < M; ++m) acc2[m] = f2_add(acc2[m], one2);
            return;
        }
        float ay, az;
        f2_unpack(v0.y, ay, az);
        const f2_t ay2 = f2_pack(ay, ay), az2 = f2_pack(az, az);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const f2_t dx = f2_sub(px2[m], v0.x);
            const f2_t dy = f2_sub(py2[m], ay2);
            const f2_t dz = f2_sub(pz2[m], az2);
            const f2_t r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
            float r0, r1;
            f2_unpack(r2, r0, r1);
            const f2_t u = f2_pack(rcp_approx(r0), rcp_approx(r1));
            const f2_t u3 = f2_mul(f2_mul(u, u), u);
            acc2[m] = f2_fma(u3, f2_fma(v1.x, u3, v1.y), acc2[m]);
        }
    };
    auto shell_atom = [&](unsigned off, int q) {
        const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(cbase + off);
        const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(cbase + off + 16);
        float ay, az;
        f2_unpack(v0.y, ay, az);
        const f2_t ay2 = f2_pack(ay, ay), az2 = f2_pack(az, az);
        float mn = INFINITY;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const f2_t dx = f2_sub(px2[m], v0.x);
            const f2_t dy = f2_sub(py2[m], ay2);
            const f2_t dz = f2_sub(pz2[m], az2);
            const f2_t r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_mul(dx, dx)));
            float r0, r1, d0, d1;
            f2_unpack(r2, r0, r1);
            const f2_t in = f2_pack(set_lt(r0, rc2f), set_lt(r1, rc2f));
            f2_unpack(f2_sub(r2, rc2), d0, d1);
            mn = fminf(mn, fminf(fabsf(d0), fabsf(d1)));
            if (PREC == PREC_COUNT) {
                acc2[m] = f2_add(acc2[m], in);
            } else {
                const f2_t u = f2_pack(rcp_approx(r0), rcp_approx(r1));
                const f2_t u3 = f2_mul(f2_mul(u, u), u);
                acc2[m] = f2_fma(f2_mul(u3, in), f2_fma(v1.x, u3, v1.y), acc2[m]);
            }
        }
        if (mn <= win) {  // rare: a pair of this atom sits near the cutoff
            rec = (rec << 10) | (unsigned)q;
            ++nrec;
        }
    };
    int q = 0;
    // the FP32 chunk sums of the inner list fold into FP64 registers, added to
    // the shared totals once (the Widom kernel has the registers for it)
    double acc64[2 * M];
#pragma unroll
    for (int m = 0; m < 2 * M; ++m) acc64[m] = 0.0;
    while (q < n_in) {
        const int qe = kComp ? min(q + PrecTraits<PREC>::inner_chunk, n_in) : n_in;
        // four atoms per iteration: sixteen independent FP32 chains for the
        // scheduler (the kernel is latency-bound at two CTAs per SM); with two
        // shell atoms per iteration and the register fold, 1.247 -> 1.207 ms
        // per 1e7 insertions on a config-1 cell
        for (; q + 3 < qe; q += 4) {
            inner_atom(wl[q]);
            inner_atom(wl[q + 1]);
            inner_atom(wl[q + 2]);
            inner_atom(wl[q + 3]);
        }
        for (; q + 1 < qe; q += 2) {
            inner_atom(wl[q]);
            inner_atom(wl[q + 1]);
        }
        if (q < qe) inner_atom(wl[q++]);
        if (kComp) fold_regs<M>(acc64, acc2);
    }
    if (kComp) {
#pragma unroll
        for (int p = 0; p < 2 * M; ++p) tot_at(s, p) += acc64[p];
    }
    q = 0;
    while (q < n_sh) {
        const int qe = kComp ? min(q + kAccChunk, n_sh) : n_sh;
        for (; q + 1 < qe; q += 2) {
            shell_atom(wl[kMaxCand - 1 - q], q);
            shell_atom(wl[kMaxCand - 2 - q], q + 1);
        }
        for (; q < qe; ++q) shell_atom(wl[kMaxCand - 1 - q], q);
        if (kComp) fold_packed<M>(s, acc2);
    }
    if (!kComp) fold_packed<M>(s, acc2);
    return nrec;
}

// Generic (per-point x, y, z) inner and shell lists, scalar FP32.
template <class Pol, int PREC>
__device__ __forceinline__ int generic_lists(EngineSmem& s, const unsigned short* wl,
                                             int n_in, int n_sh, float rc2f, float win,
                                             Lane<Pol, PREC>& L, unsigned& rec) {
    constexpr int P = Pol::kP;
    constexpr bool kComp = PrecTraits<PREC>::comp;
    float acc[P];
#pragma unroll
    for (int p = 0; p < P; ++p) acc[p] = 0.f;
    int q = 0;
    while (q < n_in) {
        const int qe = kComp ? min(q + PrecTraits<PREC>::inner_chunk, n_in) : n_in;
#pragma unroll 2
        for (; q < qe; ++q) {
            const Cand& cd = *reinterpret_cast<const Cand*>(
                reinterpret_cast<const char*>(s.cand) + wl[q]);
            const float4 v0 = *reinterpret_cast<const float4*>(&cd.ax);   // x - y z
            const float4 v1 = *reinterpret_cast<const float4*>(&cd.c12);  // C12 - -C6 -
#pragma unroll
            for (int p = 0; p < P; ++p) {
                if (PREC == PREC_COUNT) {
                    acc[p] += 1.0f;
                } else {
                    const float r2 = r2_generic(L.px[p], L.py[p], L.pz[p], v0.x, v0.z, v0.w);
                    const float u = rcp_approx(r2);
                    const float u3 = __fmul_rn(__fmul_rn(u, u), u);
                    acc[p] = __fmaf_rn(u3, __fmaf_rn(v1.x, u3, v1.z), acc[p]);
                }
            }
        }
        if (kComp) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                tot_at(s, p) += (double)acc[p];
                acc[p] = 0.f;
            }
        }
    }
    int nrec = 0;
    rec = 0;
    q = 0;
    while (q < n_sh) {
        const int qe = kComp ? min(q + kAccChunk, n_sh) : n_sh;
#pragma unroll 2
        for (; q < qe; ++q) {
            const Cand& cd = *reinterpret_cast<const Cand*>(
                reinterpret_cast<const char*>(s.cand) + wl[kMaxCand - 1 - q]);
            const float4 v0 = *reinterpret_cast<const float4*>(&cd.ax);   // x - y z
            const float4 v1 = *reinterpret_cast<const float4*>(&cd.c12);  // C12 - -C6 -
            float mn = INFINITY;
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const float r2 = r2_generic(L.px[p], L.py[p], L.pz[p], v0.x, v0.z, v0.w);
                const float dd = __fsub_rn(r2, rc2f);
                if (PREC == PREC_COUNT) {
                    if (dd < 0.f) acc[p] += 1.0f;
                } else {
                    const float u = rcp_approx(r2);
                    const float u3 = __fmul_rn(__fmul_rn(u, u), u);
                    if (dd < 0.f) acc[p] = __fmaf_rn(u3, __fmaf_rn(v1.x, u3, v1.z), acc[p]);
                }
                mn = fminf(mn, fabsf(dd));
            }
            if (mn <= win) {  // rare: a pair of this atom sits near the cutoff
                rec = (rec << 10) | (unsigned)q;
                ++nrec;
            }
        }
        if (kComp) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                tot_at(s, p) += (double)acc[p];
                acc[p] = 0.f;
            }
        }
    }
    if (!kComp) {
#pragma unroll
        for (int p = 0; p < P; ++p) tot_at(s, p) += (double)acc[p];
    }
    return nrec;
}

// Exact re-decision of the borderline shell pairs: a pair whose FP32 r^2 is
// within `win` of fl32(rc^2) is decided by exact_in_cutoff, and its term
// added or removed where the FP32 decision differed. The shell loops record
// the list positions of the atoms with such a pair (the last kRec of them,
// 10 bits each, in `rec`); past kRec records the whole shell list is
// re-examined. Kept out of line: it runs for a few
// lanes of some warps.
template <class Pol, int PREC>
static __device__ __noinline__ void recheck_borderline(EngineSmem& s, const Pol& pol,
                                                       const FwDev& fw, const CutoffConsts& cc,
                                                       const unsigned short* wl, int n_sh,
                                                       float win, int nrec, unsigned rec,
                                                       const Lane<Pol, PREC>& L) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const float rc2f = cc.rc2f;
    const bool all = nrec > kRec;
    const int nq = all ? n_sh : nrec;
    // ascending list positions either way (the latest record sits in the low
    // bits), so the corrections of a point add up in one order whichever
    // points share its thread: an energy depends only on its warp's and CTA's
    // point sets, not on where in the warp the point sits
    for (int r = 0; r < nq; ++r) {
        const int q = all ? r : (int)((rec >> (10 * (nq - 1 - r))) & 1023u);
        const unsigned off = wl[kMaxCand - 1 - q];
        const Cand& cd = s.cand[off >> 5];
        const float ss = Pol::kLattice ? ss_lattice(L.py[0], L.pz[0], cd.ay, cd.az) : 0.f;
#pragma unroll 1
        for (int p = 0; p < Pol::kP; ++p) {
            if (!(L.vmask & (1u << p))) continue;
            const float r2 =
                Pol::kLattice ? r2_lattice(L.px[p], cd.ax, ss)
                              : r2_generic(L.px[p], L.py[Pol::kLattice ? 0 : p],
                                           L.pz[Pol::kLattice ? 0 : p], cd.ax, cd.ay, cd.az);
            const float dd = __fsub_rn(r2, rc2f);
            if (fabsf(dd) <= win) {
                double f[3];
                pol.point(w, lane, p, f);
                const bool ex = exact_in_cutoff(fw, f, s.cid[off >> 5], cc.r2min);
                if (ex != (dd < 0.f)) {
                    const float e = PREC == PREC_COUNT ? 1.0f : pair_term(r2, cd.c12, cd.nc6);
                    tot_at(s, p) += ex ? (double)e : -(double)e;
                }
            }
        }
    }
}

template <class Pol, int PREC>
__device__ __forceinline__ void warp_flush_body(EngineSmem& s, const Pol& pol, const FwDev& fw,
                                                const CutoffConsts& cc, int n_cand,
                                                Lane<Pol, PREC>& L) {
    constexpr int P = Pol::kP;
    constexpr bool kNear = PrecTraits<PREC>::near64;
    constexpr bool kF64 = PrecTraits<PREC>::fp64;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (!L.warp_live) return;
    unsigned short* wl = s.wl[w];
    unsigned short* wn = s.wn[w];
    // --- split candidates into inner / shell (/ near) lists for this warp's box
    int n_in = 0, n_sh = 0, n_ni = 0, n_ns = 0;
    const unsigned lt = (1u << lane) - 1u;
    const float rnear2 = kNearR * kNearR;
    const float wl0x = s.wbox[w][0], wl0y = s.wbox[w][1], wl0z = s.wbox[w][2];
    const float wh0x = s.wbox[w][3], wh0y = s.wbox[w][4], wh0z = s.wbox[w][5];
    for (int base = 0; base < n_cand; base += 32) {
        const int c = base + lane;
        bool in = false, sh = false, nr = false;
        if (c < n_cand) {
            const float4 a = *reinterpret_cast<const float4*>(&s.cand[c].ax);
            const float ax = a.x, ay = a.z, az = a.w;
            const float ex = fmaxf(0.f, fmaxf(wl0x - ax, ax - wh0x));
            const float ey = fmaxf(0.f, fmaxf(wl0y - ay, ay - wh0y));
            const float ez = fmaxf(0.f, fmaxf(wl0z - az, az - wh0z));
            const float dmin2 = ex * ex + ey * ey + ez * ez;
            const float fx = fmaxf(fabsf(ax - wl0x), fabsf(ax - wh0x));
            const float fy = fmaxf(fabsf(ay - wl0y), fabsf(ay - wh0y));
            const float fz = fmaxf(fabsf(az - wl0z), fabsf(az - wh0z));
            const float dmax2 = fx * fx + fy * fy + fz * fz;
            in = dmax2 < cc.rin2;
            sh = !in && dmin2 < cc.rout2;
            nr = kNear && dmin2 < rnear2;
        }
        const unsigned short off = (unsigned short)(c * (int)sizeof(Cand));
        if (kNear) {
            // near atoms inside the cutoff for every point of the warp go to the
            // front of wn, near atoms crossing it (large warp boxes) to the back;
            // past kNearCap entries they stay on the FP32 lists
            const bool ni = nr && in, ns = nr && sh;
            const unsigned bni = __ballot_sync(0xffffffffu, ni);
            const unsigned bns = __ballot_sync(0xffffffffu, ns);
            const int room = kNearCap - n_ni - n_ns;
            const int ti = min(__popc(bni), room);
            const int ts = min(__popc(bns), room - ti);
            const int ai = __popc(bni & lt), as = __popc(bns & lt);
            if (ni && ai < ti) {
                wn[n_ni + ai] = off;
                in = false;
            }
            if (ns && as < ts) {
                wn[kNearCap - 1 - (n_ns + as)] = off;
                sh = false;
            }
            n_ni += ti;
            n_ns += ts;
        }
        const unsigned bi = __ballot_sync(0xffffffffu, in);
        const unsigned bs = __ballot_sync(0xffffffffu, sh);
        if (in) wl[n_in + __popc(bi & lt)] = off;
        if (sh) wl[kMaxCand - 1 - (n_sh + __popc(bs & lt))] = off;
        n_in += __popc(bi);
        n_sh += __popc(bs);
    }
    __syncwarp();

    const float rc2f = cc.rc2f;
    float win;
    {
        int e;
        frexpf(rc2f, &e);
        win = ldexpf((float)L.bul, e - 24);
    }

    // FP64 positions of this lane's points relative to the CTA centre
    // (FP64 paths only).
    auto point64 = [&](int p, double& qx, double& qy, double& qz) {
        double x, y, z, o0, o1, o2;
        pol.cart(fw.r, w, lane, p, x, y, z);
        cta_centre(s, o0, o1, o2);
        qx = x - o0;
        qy = y - o1;
        qz = z - o2;
    };

    int nrec = 0;
    unsigned rec = 0;
    if (kF64) {
        // every inner pair in FP64; shell pairs decided as below, term in FP64
        double o0, o1, o2;
        cta_centre(s, o0, o1, o2);
#pragma unroll 1
        for (int p = 0; p < P; ++p) {
            double qx, qy, qz;
            point64(p, qx, qy, qz);
            double acc = 0.0;
            for (int q = 0; q < n_in; ++q)
                acc += pair64(atom64(fw, s.cid[wl[q] >> 5], o0, o1, o2), qx, qy, qz, cc.r2min);
            double f[3];
            pol.point(w, lane, p, f);
            for (int q = 0; q < n_sh; ++q) {
                const unsigned off = wl[kMaxCand - 1 - q];
                const Cand& cd = s.cand[off >> 5];
                const float r2 = Pol::kLattice
                                     ? r2_lattice(L.px[p], cd.ax, ss_lattice(L.py[0], L.pz[0],
                                                                             cd.ay, cd.az))
                                     : r2_generic(L.px[p], L.py[Pol::kLattice ? 0 : p],
                                                  L.pz[Pol::kLattice ? 0 : p], cd.ax, cd.ay,
                                                  cd.az);
                const float dd = __fsub_rn(r2, rc2f);
                bool inside = dd < 0.f;
                if (fabsf(dd) <= win) inside = exact_in_cutoff(fw, f, s.cid[off >> 5], cc.r2min);
                if (inside)
                    acc += pair64(atom64(fw, s.cid[off >> 5], o0, o1, o2), qx, qy, qz, cc.r2min);
            }
            tot_at(s, p) += acc;
        }
        return;
    }

    if (Pol::kLattice) {
        lattice_inner<Pol, PREC>(s, wl, n_in, L);
        nrec = lattice_shell<Pol, PREC>(s, wl, n_sh, rc2f, win, L, rec);
    } else {
        nrec = (Pol::kP % 2 == 0)
                   ? generic_packed_lists<Pol, PREC>(s, wl, n_in, n_sh, rc2f, win, L, rec)
                   : generic_lists<Pol, PREC>(s, wl, n_in, n_sh, rc2f, win, L, rec);
    }

    // --- exact re-decision of borderline shell pairs (rare); lanes without a
    // flagged point idle through it
    if (nrec > 0) recheck_borderline<Pol, PREC>(s, pol, fw, cc, wl, n_sh, win, nrec, rec, L);
    // --- near lists in FP64: exact positions (FP64 images and points relative
    // to the CTA centre) and FP64 (C12, C6). Atom-outer order: one atom's loads
    // serve kNearP of the lane's points per pass.
    if (kNear && n_ni + n_ns > 0) {
        // lattice lanes take all P points in one pass (their FP32 list state is
        // dead by now, so the FP64 point state fits the 80 registers); generic
        // points, with their own y and z each, take passes of 4
        constexpr int kNearP = Pol::kLattice ? P : (P < 4 ? P : 4);
        double o0, o1, o2;
        cta_centre(s, o0, o1, o2);
#pragma unroll 1
        for (int p0 = 0; p0 < P; p0 += kNearP) {
            double qx[kNearP], qy[Pol::kLattice ? 1 : kNearP], qz[Pol::kLattice ? 1 : kNearP];
            double nacc[kNearP];
#pragma unroll
            for (int p = 0; p < kNearP; ++p) {
                double y, z;
                point64(p0 + p, qx[p], y, z);
                if (!Pol::kLattice || p == 0) {
                    qy[Pol::kLattice ? 0 : p] = y;
                    qz[Pol::kLattice ? 0 : p] = z;
                }
                nacc[p] = 0.0;
            }
            // atoms inside the cutoff for every point of the warp: no test
            // Widom points: the next atom's FP64 data is loaded while this one's
            // terms run (the 128-register Widom kernel has room for it; at the
            // grid kernels' 80 registers it costs more than it hides)
            constexpr bool kPrefetch = !Pol::kLattice;
            Atom64 nxt = (kPrefetch && n_ni > 0) ? atom64(fw, s.cid[wn[0] >> 5], o0, o1, o2)
                                                 : Atom64{};
            for (int q = 0; q < n_ni; ++q) {
                Atom64 a;
                if (kPrefetch) {
                    a = nxt;
                    if (q + 1 < n_ni) nxt = atom64(fw, s.cid[wn[q + 1] >> 5], o0, o1, o2);
                } else {
                    a = atom64(fw, s.cid[wn[q] >> 5], o0, o1, o2);
                }
                if (Pol::kLattice) {
                    // a lattice lane's points share y and z: dy^2 + dz^2 once per atom
                    const double dy = qy[0] - a.y, dz = qz[0] - a.z;
                    const double yzc = fma(dz, dz, fma(dy, dy, cc.r2min));
#pragma unroll
                    for (int p = 0; p < kNearP; ++p)
                        nacc[p] = near_acc64(nacc[p], qx[p] - a.x, yzc, a.c12, a.c6);
                } else {
#pragma unroll
                    for (int p = 0; p < kNearP; ++p) {
                        const double dy = qy[p] - a.y, dz = qz[p] - a.z;
                        nacc[p] = near_acc64(nacc[p], qx[p] - a.x,
                                             fma(dz, dz, fma(dy, dy, cc.r2min)), a.c12, a.c6);
                    }
                }
            }
            // atoms crossing the cutoff inside the warp box (boxes wider than
            // rc - kNearR: coarse grids, sparse Widom bins): the cutoff decided per
            // pair on the FP64 r^2. It differs from the reference's FP64 r^2 (cell
            // frame, its own rounding) by far less than 1e-12 rc^2, so outside that
            // window both decide alike and inside it exact_in_cutoff decides.
            const double rc2lo = fw.rc2 * (1.0 - 1e-12), rc2hi = fw.rc2 * (1.0 + 1e-12);
            for (int q = 0; q < n_ns; ++q) {
                const int gid = s.cid[wn[kNearCap - 1 - q] >> 5];
                const Atom64 a = atom64(fw, gid, o0, o1, o2);
#pragma unroll 1
                for (int p = 0; p < kNearP; ++p) {
                    if (!(L.vmask & (1u << (p0 + p)))) continue;  // never stored
                    const double dy = qy[Pol::kLattice ? 0 : p] - a.y;
                    const double dz = qz[Pol::kLattice ? 0 : p] - a.z;
                    const double dx = qx[p] - a.x;
                    const double r2 = fmax(fma(dx, dx, fma(dz, dz, dy * dy)), cc.r2min);
                    bool inside = r2 < rc2lo;
                    if (!inside && r2 < rc2hi) {
                        double f[3];
                        pol.point(w, lane, p0 + p, f);
                        inside = exact_in_cutoff(fw, f, gid, cc.r2min);
                    }
                    if (inside) {
                        const double u = rcp64_nr(r2);
                        const double u3 = u * u * u;
                        nacc[p] = fma(u3, fma(a.c12, u3, -a.c6), nacc[p]);
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < kNearP; ++p) tot_at(s, p0 + p) += nacc[p];
        }
    }
}

// Lattice (grid) flushes run out of line: the producer's loop state (box,
// cell ranges, counters) is saved once around the call instead of staying
// live in registers through the pair loops (at the 80-register limit of three
// CTAs per SM that took the 256-framework batch from 370 to 357 ms). The
// Widom kernel (128 registers, generic points) is faster with the flush
// inlined: 1.28 ms per 1e7 insertions against 1.61 ms out of line; out of
// line at 80 registers and three CTAs per SM (P = 4, 6 or 8) it took
// 1.42-1.51 ms.
template <class Pol, int PREC>
static __device__ __noinline__ void warp_flush_call(EngineSmem& s, const Pol& pol,
                                                    const FwDev& fw, const CutoffConsts& cc,
                                                    int n_cand, Lane<Pol, PREC>& L) {
    warp_flush_body<Pol, PREC>(s, pol, fw, cc, n_cand, L);
}

template <class Pol, int PREC>
__device__ __forceinline__ void warp_flush(EngineSmem& s, const Pol& pol, const FwDev& fw,
                                           const CutoffConsts& cc, int n_cand,
                                           Lane<Pol, PREC>& L) {
    if constexpr (Pol::kLattice)
        warp_flush_call<Pol, PREC>(s, pol, fw, cc, n_cand, L);
    else
        warp_flush_body<Pol, PREC>(s, pol, fw, cc, n_cand, L);
}

template <class Pol, int PREC>
__device__ void process_cta(EngineSmem& s, const Pol& pol, const FwDev& fw,
                            const CutoffConsts& cc) {
    constexpr int P = Pol::kP;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    Lane<Pol, PREC> L;

    // 1. the CTA box: FP64 bounding box of the valid points
    L.vmask = 0;
    double mn0 = INFINITY, mn1 = INFINITY, mn2 = INFINITY;
    double mx0 = -INFINITY, mx1 = -INFINITY, mx2 = -INFINITY;
#pragma unroll
    for (int p = 0; p < P; ++p) {
        double x, y, z;
        const bool ok = pol.cart(fw.r, w, lane, p, x, y, z);
        if (ok) {
            L.vmask |= 1u << p;
            mn0 = fmin(mn0, x); mn1 = fmin(mn1, y); mn2 = fmin(mn2, z);
            mx0 = fmax(mx0, x); mx1 = fmax(mx1, y); mx2 = fmax(mx2, z);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn0 = fmin(mn0, __shfl_xor_sync(0xffffffffu, mn0, o));
        mn1 = fmin(mn1, __shfl_xor_sync(0xffffffffu, mn1, o));
        mn2 = fmin(mn2, __shfl_xor_sync(0xffffffffu, mn2, o));
        mx0 = fmax(mx0, __shfl_xor_sync(0xffffffffu, mx0, o));
        mx1 = fmax(mx1, __shfl_xor_sync(0xffffffffu, mx1, o));
        mx2 = fmax(mx2, __shfl_xor_sync(0xffffffffu, mx2, o));
    }
    L.warp_live = __any_sync(0xffffffffu, L.vmask != 0);
    if (lane == 0) {
        s.red[w][0] = mn0; s.red[w][1] = mn1; s.red[w][2] = mn2;
        s.red[w][3] = mx0; s.red[w][4] = mx1; s.red[w][5] = mx2;
    }
    __syncthreads();
    if (tid < 6) {
        double v = s.red[0][tid];
        for (int k = 1; k < kWarps; ++k)
            v = (tid < 3) ? fmin(v, s.red[k][tid]) : fmax(v, s.red[k][tid]);
        s.box[tid] = v;
    }
    __syncthreads();
    const double lo0 = s.box[0], lo1 = s.box[1], lo2 = s.box[2];
    const double hi0 = s.box[3], hi1 = s.box[4], hi2 = s.box[5];
    __syncthreads();
    if (!(lo0 <= hi0)) return;  // no valid point in this CTA
    double o0, o1, o2;
    cta_centre(s, o0, o1, o2);
    L.bul = borderline_ulps(
        cc.rc, cc.rc2f,
        sqrt((hi0 - lo0) * (hi0 - lo0) + (hi1 - lo1) * (hi1 - lo1) + (hi2 - lo2) * (hi2 - lo2)));

    // 2. local FP32 coordinates and the warp box (a lattice lane's points
    // share y and z bit for bit: R[1][0] = R[2][0] = 0)
    {
        float wl0x = INFINITY, wl0y = INFINITY, wl0z = INFINITY;
        float wh0x = -INFINITY, wh0y = -INFINITY, wh0z = -INFINITY;
#pragma unroll
        for (int p = 0; p < P; ++p) {
            double x, y, z;
            pol.cart(fw.r, w, lane, p, x, y, z);
            const float fx = (float)(x - o0), fy = (float)(y - o1), fz = (float)(z - o2);
            L.px[p] = fx;
            if (!Pol::kLattice || p == 0) {
                L.py[Pol::kLattice ? 0 : p] = fy;
                L.pz[Pol::kLattice ? 0 : p] = fz;
            }
            tot_at(s, p) = 0.0;
            if (L.vmask & (1u << p)) {
                wl0x = fminf(wl0x, fx); wl0y = fminf(wl0y, fy); wl0z = fminf(wl0z, fz);
                wh0x = fmaxf(wh0x, fx); wh0y = fmaxf(wh0y, fy); wh0z = fmaxf(wh0z, fz);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            wl0x = fminf(wl0x, __shfl_xor_sync(0xffffffffu, wl0x, o));
            wl0y = fminf(wl0y, __shfl_xor_sync(0xffffffffu, wl0y, o));
            wl0z = fminf(wl0z, __shfl_xor_sync(0xffffffffu, wl0z, o));
            wh0x = fmaxf(wh0x, __shfl_xor_sync(0xffffffffu, wh0x, o));
            wh0y = fmaxf(wh0y, __shfl_xor_sync(0xffffffffu, wh0y, o));
            wh0z = fmaxf(wh0z, __shfl_xor_sync(0xffffffffu, wh0z, o));
        }
        if (lane == 0) {
            s.wbox[w][0] = wl0x; s.wbox[w][1] = wl0y; s.wbox[w][2] = wl0z;
            s.wbox[w][3] = wh0x; s.wbox[w][4] = wh0y; s.wbox[w][5] = wh0z;
        }
        __syncwarp();
    }

// ER_BULK=1 (a build option: `make -C emptyroom_b200/csrc clean all cli
// ER_BULK=1`) selects the producer whose cell-row image ranges arrive in
// shared memory by bulk copies of the TMA engine (cp.async.bulk, 256 images
// per stage, two stages in flight, each completing on an mbarrier whose wait
// is bounded). Measured on the 256-framework batch it is slower than the
// default producer (per-thread loads of the same images): 352.1 against
// 341.6 ms in the default mode, 305.8 against 297.3 ms in ER_PREC_COMP, a
// Widom call of 1e7 insertions 1.741 against 1.727 ms -- each stage adds a
// block-wide wait, and the staging state raises the producer's register
// spills (grid_persistent_kernel<3>: 364 / 1000 bytes of spill stores / loads
// against 280 / 584).
#ifndef ER_BULK
#define ER_BULK 0
#endif
#if ER_BULK
    // staging barriers of this pass (initialised here, invalidated at its end)
    if (tid == 0) {
        mbar_init(&s.mbar[0]);
        mbar_init(&s.mbar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
#endif
#if ER_BULK
    unsigned mph = 0;    // phase parity of each staging barrier
#endif
    bool fault = false;  // a staging wait gave up
    // 3. producer: rows of cells around the CTA box, streamed into shared memory
    const double R = cc.rcm, R2 = R * R;
    const float R2f = (float)R2;
    const float b0x = (float)(lo0 - o0), b0y = (float)(lo1 - o1), b0z = (float)(lo2 - o2);
    const float b1x = (float)(hi0 - o0), b1y = (float)(hi1 - o1), b1z = (float)(hi2 - o2);
    int c0[3], c1[3];
    {
        const double lov[3] = {lo0, lo1, lo2}, hiv[3] = {hi0, hi1, hi2};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            c0[d] = max(0, (int)floor((lov[d] - R - fw.cell_lo[d]) * fw.inv_h));
            c1[d] = min(fw.nc[d] - 1, (int)floor((hiv[d] + R - fw.cell_lo[d]) * fw.inv_h));
        }
    }
    int n_cand = 0;
    if (c0[0] <= c1[0] && c0[1] <= c1[1] && c0[2] <= c1[2]) {
        const int nyr = c1[1] - c0[1] + 1, nzr = c1[2] - c0[2] + 1;
        const int nrows = nyr * nzr;
        for (int rb = 0; rb < nrows; rb += kRowChunk) {
            const int r = rb + tid;
            int beg = 0, len = 0;
            if (r < nrows) {
                const int ry = c0[1] + r % nyr, rz = c0[2] + r / nyr;
                const double ylo = fw.cell_lo[1] + ry * fw.h, yhi = ylo + fw.h;
                const double zlo = fw.cell_lo[2] + rz * fw.h, zhi = zlo + fw.h;
                const double dy = fmax(0.0, fmax(ylo - hi1, lo1 - yhi));
                const double dz = fmax(0.0, fmax(zlo - hi2, lo2 - zhi));
                const double d2 = dy * dy + dz * dz;
                if (d2 < R2) {
                    const double ex = sqrt(R2 - d2);
                    const int xa = max(c0[0], (int)floor((lo0 - ex - fw.cell_lo[0]) * fw.inv_h));
                    const int xb = min(c1[0], (int)floor((hi0 + ex - fw.cell_lo[0]) * fw.inv_h));
                    if (xa <= xb) {
                        const int rowb = (rz * fw.nc[1] + ry) * fw.nc[0];
                        beg = fw.cell_start[rowb + xa];
                        len = fw.cell_start[rowb + xb + 1] - beg;
                    }
                }
            }
            int tot;
            const int off = block_exscan(len, s.warp_tot, &tot);
            s.row_beg[tid] = beg;
            s.row_off[tid] = off;
            __syncthreads();
            const int nr = min(kRowChunk, nrows - rb);
#if ER_BULK
            // the rows' image ranges arrive by bulk copies, kThreads images
            // per stage, two stages in flight in the staging area (the per-warp
            // lists, unused while the producer runs)
            double4* stg = reinterpret_cast<double4*>(&s.wl[0][0]);
            const int nst = (tot + kThreads - 1) / kThreads;
            auto issue = [&](int k) {
                const int b = k & 1;
                const int lo = k * kThreads, hi = min(tot, lo + kThreads);
                if (tid == 0) mbar_expect_tx(&s.mbar[b], (unsigned)(hi - lo) * 32u);
                const int a = max(lo, off), e = min(hi, off + len);
                if (a < e)
                    bulk_g2s(stg + b * kThreads + (a - lo), fw.img_xyz + beg + (a - off),
                             (unsigned)(e - a) * 32u, &s.mbar[b]);
            };
            if (nst > 0) issue(0);
            for (int k = 0; k < nst; ++k) {
                const int b = k & 1;
                if (k + 1 < nst) issue(k + 1);
                fault |= !mbar_wait(&s.mbar[b], (mph >> b) & 1u);
                mph ^= 1u << b;
                const int c = k * kThreads + tid;
                int pass = 0, g = 0;
                float ax = 0.f, ay = 0.f, az = 0.f, c12 = 0.f, nc6 = 0.f;
                if (c < tot) {
                    const double4 ap = stg[b * kThreads + tid];
                    ax = (float)(ap.x - o0);
                    ay = (float)(ap.y - o1);
                    az = (float)(ap.z - o2);
                    const float ddx = fmaxf(0.f, fmaxf(b0x - ax, ax - b1x));
                    const float ddy = fmaxf(0.f, fmaxf(b0y - ay, ay - b1y));
                    const float ddz = fmaxf(0.f, fmaxf(b0z - az, az - b1z));
                    pass = (ddx * ddx + ddy * ddy + ddz * ddz) < R2f;
                    if (pass) {
                        int a = 0, bb = nr - 1;
                        while (a < bb) {
                            const int mid = (a + bb + 1) >> 1;
                            if (s.row_off[mid] <= c) a = mid; else bb = mid - 1;
                        }
                        g = s.row_beg[a] + (c - s.row_off[a]);
                        const float2 pr = fw.img_par[g];
                        c12 = pr.x;
                        nc6 = pr.y;
                    }
                }
                int npass;
                const int pos = block_exscan(pass, s.warp_tot, &npass);
                if (n_cand + npass > kMaxCand) {
                    // the flush writes the staging area: the next stage lands
                    // first and is copied again after it
                    if (k + 1 < nst) {
                        fault |= !mbar_wait(&s.mbar[b ^ 1], (mph >> (b ^ 1)) & 1u);
                        mph ^= 1u << (b ^ 1);
                    }
                    __syncthreads();
                    warp_flush<Pol, PREC>(s, pol, fw, cc, n_cand, L);
                    __syncthreads();
                    n_cand = 0;
                    if (k + 1 < nst) issue(k + 1);
                }
                if (pass) {
                    Cand& dst = s.cand[n_cand + pos];
                    *reinterpret_cast<float4*>(&dst.ax) = make_float4(ax, ax, ay, az);
                    *reinterpret_cast<float4*>(&dst.c12) = make_float4(c12, c12, nc6, nc6);
                    s.cid[n_cand + pos] = g;
                }
                n_cand += npass;
            }
#else
            for (int cb = 0; cb < tot; cb += kThreads) {
                const int c = cb + tid;
                int pass = 0, g = 0;
                float ax = 0.f, ay = 0.f, az = 0.f, c12 = 0.f, nc6 = 0.f;
                if (c < tot) {
                    int a = 0, b = nr - 1;
                    while (a < b) {
                        const int mid = (a + b + 1) >> 1;
                        if (s.row_off[mid] <= c) a = mid; else b = mid - 1;
                    }
                    g = s.row_beg[a] + (c - s.row_off[a]);
                    const double4 ap = fw.img_xyz[g];
                    ax = (float)(ap.x - o0);
                    ay = (float)(ap.y - o1);
                    az = (float)(ap.z - o2);
                    const float ddx = fmaxf(0.f, fmaxf(b0x - ax, ax - b1x));
                    const float ddy = fmaxf(0.f, fmaxf(b0y - ay, ay - b1y));
                    const float ddz = fmaxf(0.f, fmaxf(b0z - az, az - b1z));
                    pass = (ddx * ddx + ddy * ddy + ddz * ddz) < R2f;
                    if (pass) {
                        const float2 pr = fw.img_par[g];
                        c12 = pr.x;
                        nc6 = pr.y;
                    }
                }
                int npass;
                const int pos = block_exscan(pass, s.warp_tot, &npass);
                if (n_cand + npass > kMaxCand) {
                    __syncthreads();
                    warp_flush<Pol, PREC>(s, pol, fw, cc, n_cand, L);
                    __syncthreads();
                    n_cand = 0;
                }
                if (pass) {
                    Cand& dst = s.cand[n_cand + pos];
                    *reinterpret_cast<float4*>(&dst.ax) = make_float4(ax, ax, ay, az);
                    *reinterpret_cast<float4*>(&dst.c12) = make_float4(c12, c12, nc6, nc6);
                    s.cid[n_cand + pos] = g;
                }
                n_cand += npass;
            }
#endif
            __syncthreads();
        }
    }
    if (n_cand > 0) {
        __syncthreads();
        warp_flush<Pol, PREC>(s, pol, fw, cc, n_cand, L);
    }
    // 4. store (nothing when a staging wait gave up: the pass is reported
    // through the fault word instead of storing energies of missing atoms)
    if (__syncthreads_or(fault)) {
        if (tid == 0 && fw.fault) atomicExch(fw.fault, 1);
        L.vmask = 0;
    }
#if ER_BULK
    if (tid == 0) {
        mbar_inval(&s.mbar[0]);
        mbar_inval(&s.mbar[1]);
    }
#endif
#pragma unroll
    for (int p = 0; p < P; ++p) {
        if (L.vmask & (1u << p)) {
            if (PrecTraits<PREC>::fp64) {
                pol.store64(w, lane, p, fmin(tot_at(s, p), (double)kEnergyCap));
            } else {
                float e = (float)tot_at(s, p);
                if (PREC != PREC_COUNT) e = fminf(e, kEnergyCap);
                pol.store(w, lane, p, e);
            }
        }
    }
    __syncthreads();
}

}  // namespace er
