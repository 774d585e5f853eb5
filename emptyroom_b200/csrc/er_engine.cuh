// er_engine.cuh -- the probe-framework Lennard-Jones pair-sum engine (sm_100a).
//
// What it computes is the sum of src/computegridsheet.h:54-92 (and the same
// sum in src/doHenry.h:70-98): at every point p, over every kept atom image
// a + T n, 4 eps s^6 (s^6 - 1) with s = sig^2 / r^2 when r^2 < rc^2.
// How it computes it is its own:
//
//  * A CTA owns up to 8 warp tasks of <= 32*P points (a lattice sub-brick of
//    the grid, or a chunk of one spatial bin of Widom insertions). The CTA box
//    is the FP64 bounding box of its points; all FP32 coordinates are relative
//    to the box centre, so FP32 never holds magnitudes above rc + box.
//  * Candidate atom images come from the framework's cell list: one contiguous
//    image range per (y, z) row of cells, with the x range of each row pruned
//    by the cutoff circle. Passing candidates are compacted in order (block
//    scans, so the order is deterministic) into shared memory as
//    (dx, dy, dz, C12) + (-C6).
//  * Each warp splits the CTA candidates against its own box into an inner
//    list (inside the cutoff for every point of the warp: no test needed) and
//    a shell list (cutoff tested per pair). Lists are u16 indices.
//  * Pair term: u = rcp(r^2) (one MUFU), u3 = u^3, E += u3 (C12 u3 - C6):
//    10 FP32-pipe instructions per pair on the inner list.
//  * Shell pairs whose FP32 r^2 lies within a proven error window of rc^2 are
//    re-decided in FP64 with the reference's own expression order, so the set
//    of summed pairs equals the FP64 reference's set exactly.
//  * Accumulation: FP32 per chunk of 64 atoms, folded into a two-float
//    (hi, lo) sum with TwoSum (ER_PREC_COMP), or plain FP32 (ER_PREC_FP32).
#pragma once
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "er_internal.h"

namespace er {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
// points per thread (P) and the CTA brick are set by the point policy (Tile)
constexpr int kWJ = 4, kWK = 8;            // lanes of a warp sub-brick along j, k
constexpr int kPMax = 8;                   // largest P any policy uses
constexpr int kMaxCand = 2048;             // CTA candidate capacity per flush
constexpr int kRowChunk = kThreads;        // cell rows examined per producer pass
constexpr int kAccChunk = 64;              // atoms per FP32 partial sum
constexpr float kEnergyCap = 1.0e30f;      // overflow cap (ER_ENERGY_CAP)

// PREC_COUNT writes the number of in-cutoff pair terms per point instead of
// the energy (same traversal; used to count the algorithmic work of a job).
// PREC_NEAR64 is PREC_COMP with the pairs of atoms within kNearR of a warp's
// box evaluated in FP64 (they carry most of |E| where terms cancel).
enum { PREC_COMP = 0, PREC_FP32 = 1, PREC_COUNT = 2, PREC_NEAR64 = 3 };

template <int PREC>
struct PrecTraits {
    static constexpr bool comp = PREC == PREC_COMP || PREC == PREC_NEAR64;
    static constexpr bool near64 = PREC == PREC_NEAR64;
};

constexpr int kNearCap = 256;     // near-list capacity per warp (overflow stays FP32)
constexpr float kNearR = 5.0f;    // near radius (A) from the warp box

// One candidate atom image in shared memory (32 bytes, so a list entry can be
// the byte offset of its record and a load needs no index arithmetic).
struct __align__(32) Cand {
    float4 p;    // (dx, dy, dz, C12), position relative to the CTA centre
    float nc6;   // -C6
    int id;      // image index (for the FP64 re-decision)
    float pad0, pad1;
};

__device__ __forceinline__ const Cand& cand_at(const Cand* base, unsigned off) {
    return *reinterpret_cast<const Cand*>(reinterpret_cast<const char*>(base) + off);
}

struct __align__(16) EngineSmem {
    Cand cand[kMaxCand];                   // CTA candidates
    unsigned short wl[kWarps][kMaxCand];   // per-warp inner (front) / shell (back) lists of
                                           // byte offsets into cand
    unsigned short wn[kWarps][kNearCap];   // per-warp near lists (PREC_NEAR64)
    int row_beg[kRowChunk];
    int row_off[kRowChunk];
    int warp_tot[kWarps];
    double red[kWarps][6];
    double box[6];
    int item;
};

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
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
// src/computegridsheet.h:61-79 evaluated in IEEE double without contraction.
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

// FP32 pair term with a fixed instruction sequence, so that a later
// re-evaluation reproduces the same bits.
__device__ __forceinline__ void pair_r2(float px, float py, float pz, const float4& a,
                                        float& r2) {
    const float dx = __fsub_rn(px, a.x);
    const float dy = __fsub_rn(py, a.y);
    const float dz = __fsub_rn(pz, a.z);
    r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}
// E_pair = u3 * t with u = 1/r^2, u3 = u^3, t = C12 u3 - C6.
__device__ __forceinline__ void pair_ut(float r2, float c12, float nc6, float& u3, float& t) {
    const float u = rcp_approx(r2);
    u3 = __fmul_rn(__fmul_rn(u, u), u);
    t = __fmaf_rn(c12, u3, nc6);
}

__device__ __forceinline__ void two_sum_into(float& hi, float& lo, float a) {
    const float s = __fadd_rn(hi, a);
    const float bp = __fsub_rn(s, hi);
    const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(a, bp));
    hi = s;
    lo = __fadd_rn(lo, e);
}

// ---------------------------------------------------------------------------
// Point sources. A policy maps (warp, lane, p) to an FP64 fractional point
// and stores its energy.

// Lattice points of one (2P) x 8 x 16 brick of a grid job: warp w owns the
// P x 4 x 8 sub-brick at ((w & 1) P, ((w >> 1) & 1) 4, (w >> 2) 8); lane l the
// (j, k) = (l / 8, l % 8) column of it and its P points along i.
template <int P_>
struct GridPolicy {
    static constexpr int kP = P_;
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
    __device__ __forceinline__ void store(int w, int lane, int p, float e) const {
        int i, j, k;
        index(w, lane, p, i, j, k);
        if (i < T->nx && j < T->ny && k < T->nz)
            T->out[(size_t)k + (size_t)j * T->nz + (size_t)i * T->ny * T->nz] = e;
    }
};

// Widom insertion points: CTA c owns sorted positions [256 P c, 256 P (c + 1))
// of `order`; warp w the 32 P positions from 256 P c + 32 P w.
template <int P_>
struct PointPolicy {
    static constexpr int kP = P_;
    const PointTask* T;
    int base, nv;
    __device__ PointPolicy(const PointTask* task, int cta)
        : T(task), base(cta * kWarps * 32 * kP), nv(*task->n_valid) {}
    __device__ __forceinline__ int slot_index(int w, int lane, int p) const {
        const int pos = base + w * (32 * kP) + p * 32 + lane;
        return pos < nv ? T->order[pos] : -1;
    }
    __device__ __forceinline__ bool point(int w, int lane, int p, double* f) const {
        int idx = slot_index(w, lane, p);
        const bool ok = idx >= 0;
        if (!ok) idx = T->order[min(base, nv - 1)];  // a finite stand-in, never stored
        f[0] = T->pts[3 * (size_t)idx];
        f[1] = T->pts[3 * (size_t)idx + 1];
        f[2] = T->pts[3 * (size_t)idx + 2];
        return ok;
    }
    __device__ __forceinline__ void store(int w, int lane, int p, float e) const {
        const int idx = slot_index(w, lane, p);
        if (idx >= 0) T->energies[idx] = e;
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

template <class Pol, int PREC>
__device__ __forceinline__ void warp_flush(EngineSmem& s, const Pol& pol, const FwDev& fw,
                                           const CutoffConsts& cc, int n_cand,
                                           const float* px, const float* py, const float* pz,
                                           float* hi, float* lo, double* nacc, float wl0x,
                                           float wl0y, float wl0z, float wh0x, float wh0y,
                                           float wh0z, bool warp_live, unsigned vmask,
                                           int bul_i) {
    constexpr bool kComp = PrecTraits<PREC>::comp;
    constexpr bool kNear = PrecTraits<PREC>::near64;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (!warp_live) return;
    unsigned short* wl = s.wl[w];
    unsigned short* wn = s.wn[w];
    // --- split candidates into inner / shell (/ near) lists for this warp's box
    int n_in = 0, n_sh = 0, n_near = 0;
    const unsigned lt = (1u << lane) - 1u;
    const float rnear2 = kNearR * kNearR;
    for (int base = 0; base < n_cand; base += 32) {
        const int c = base + lane;
        bool in = false, sh = false, nr = false;
        if (c < n_cand) {
            const float4 a = s.cand[c].p;
            const float ex = fmaxf(0.f, fmaxf(wl0x - a.x, a.x - wh0x));
            const float ey = fmaxf(0.f, fmaxf(wl0y - a.y, a.y - wh0y));
            const float ez = fmaxf(0.f, fmaxf(wl0z - a.z, a.z - wh0z));
            const float dmin2 = ex * ex + ey * ey + ez * ez;
            const float fx = fmaxf(fabsf(a.x - wl0x), fabsf(a.x - wh0x));
            const float fy = fmaxf(fabsf(a.y - wl0y), fabsf(a.y - wh0y));
            const float fz = fmaxf(fabsf(a.z - wl0z), fabsf(a.z - wh0z));
            const float dmax2 = fx * fx + fy * fy + fz * fz;
            in = dmax2 < cc.rin2;
            sh = !in && dmin2 < cc.rout2;
            nr = kNear && in && dmin2 < rnear2;
        }
        const unsigned short off = (unsigned short)(c * (int)sizeof(Cand));
        if (kNear) {
            const unsigned bn = __ballot_sync(0xffffffffu, nr);
            const int at = n_near + __popc(bn & lt);
            if (nr && at >= kNearCap) nr = false;  // overflow: stays on the FP32 inner list
            if (nr) {
                wn[at] = off;
                in = false;
            }
            n_near = min(kNearCap, n_near + __popc(bn));
        }
        const unsigned bi = __ballot_sync(0xffffffffu, in);
        const unsigned bs = __ballot_sync(0xffffffffu, sh);
        if (in) wl[n_in + __popc(bi & lt)] = off;
        if (sh) wl[kMaxCand - 1 - (n_sh + __popc(bs & lt))] = off;
        n_in += __popc(bi);
        n_sh += __popc(bs);
    }
    __syncwarp();

    // --- inner list: every pair is inside the cutoff
    float acc[Pol::kP];
#pragma unroll
    for (int p = 0; p < Pol::kP; ++p) acc[p] = 0.f;
    int q = 0;
    while (q < n_in) {
        const int qe = kComp ? min(q + kAccChunk, n_in) : n_in;
#pragma unroll 2
        for (; q < qe; ++q) {
            const Cand& cd = cand_at(s.cand, wl[q]);
            const float4 a = cd.p;
            const float nc6 = cd.nc6;
#pragma unroll
            for (int p = 0; p < Pol::kP; ++p) {
                if (PREC == PREC_COUNT) {
                    acc[p] += 1.0f;
                } else {
                    float r2, u3, t;
                    pair_r2(px[p], py[p], pz[p], a, r2);
                    pair_ut(r2, a.w, nc6, u3, t);
                    acc[p] = __fmaf_rn(u3, t, acc[p]);
                }
            }
        }
        if (kComp) {
#pragma unroll
            for (int p = 0; p < Pol::kP; ++p) {
                two_sum_into(hi[p], lo[p], acc[p]);
                acc[p] = 0.f;
            }
        }
    }
    // --- shell list: cutoff tested per pair, borderline pairs flagged.
    // dd = r^2 - fl32(rc^2) is exact wherever |dd| is near the window
    // (Sterbenz), so |dd| <= win selects exactly the pairs within bul ulps.
    const float rc2f = cc.rc2f;
    float win;
    {
        int e;
        frexpf(rc2f, &e);
        win = ldexpf((float)bul_i, e - 24);
    }
    bool bf[Pol::kP];
#pragma unroll
    for (int p = 0; p < Pol::kP; ++p) bf[p] = false;
    q = 0;
    while (q < n_sh) {
        const int qe = kComp ? min(q + kAccChunk, n_sh) : n_sh;
#pragma unroll 2
        for (; q < qe; ++q) {
            const Cand& cd = cand_at(s.cand, wl[kMaxCand - 1 - q]);
            const float4 a = cd.p;
            const float nc6 = cd.nc6;
#pragma unroll
            for (int p = 0; p < Pol::kP; ++p) {
                float r2, u3, t;
                pair_r2(px[p], py[p], pz[p], a, r2);
                const float dd = __fsub_rn(r2, rc2f);
                if (PREC == PREC_COUNT) {
                    if (dd < 0.f) acc[p] += 1.0f;
                } else {
                    pair_ut(r2, a.w, nc6, u3, t);
                    if (dd < 0.f) acc[p] = __fmaf_rn(u3, t, acc[p]);
                }
                bf[p] = bf[p] || (fabsf(dd) <= win);
            }
        }
        if (kComp) {
#pragma unroll
            for (int p = 0; p < Pol::kP; ++p) {
                two_sum_into(hi[p], lo[p], acc[p]);
                acc[p] = 0.f;
            }
        }
    }
    if (!kComp) {
#pragma unroll
        for (int p = 0; p < Pol::kP; ++p) hi[p] = __fadd_rn(hi[p], acc[p]);
    }
    // --- exact re-decision of borderline shell pairs (rare)
    unsigned bflag = 0;
#pragma unroll
    for (int p = 0; p < Pol::kP; ++p) bflag |= bf[p] ? (1u << p) : 0u;
    bflag &= vmask;
    if (__any_sync(0xffffffffu, bflag != 0)) {
        for (int p = 0; p < Pol::kP; ++p) {
            if (!(bflag & (1u << p))) continue;
            double f[3];
            pol.point(w, lane, p, f);
            float corr = 0.f;
            for (int qq = 0; qq < n_sh; ++qq) {
                const Cand& cd = cand_at(s.cand, wl[kMaxCand - 1 - qq]);
                const float4 a = cd.p;
                float r2;
                pair_r2(px[p], py[p], pz[p], a, r2);
                const float dd = __fsub_rn(r2, rc2f);
                if (fabsf(dd) <= win) {
                    const bool ex = exact_in_cutoff(fw, f, cd.id, cc.r2min);
                    if (ex != (dd < 0.f)) {
                        float e = 1.0f;
                        if (PREC != PREC_COUNT) {
                            float u3, t;
                            pair_ut(r2, a.w, cd.nc6, u3, t);
                            e = __fmul_rn(u3, t);
                        }
                        corr = ex ? __fadd_rn(corr, e) : __fsub_rn(corr, e);
                    }
                }
            }
            if (kComp) two_sum_into(hi[p], lo[p], corr);
            else hi[p] = __fadd_rn(hi[p], corr);
        }
    }
    // --- near list in FP64: exact positions (FP64 images and points relative
    // to the CTA centre) and FP64 (C12, C6); all near atoms are inner atoms.
    if (kNear && n_near > 0) {
        const double o0 = 0.5 * (s.box[0] + s.box[3]);
        const double o1 = 0.5 * (s.box[1] + s.box[4]);
        const double o2 = 0.5 * (s.box[2] + s.box[5]);
        double qx[Pol::kP], qy[Pol::kP], qz[Pol::kP];
#pragma unroll
        for (int p = 0; p < Pol::kP; ++p) {
            double f[3], x, y, z;
            pol.point(w, lane, p, f);
            frac_to_cart(fw.t, f[0], f[1], f[2], x, y, z);
            qx[p] = x - o0;
            qy[p] = y - o1;
            qz[p] = z - o2;
        }
        for (int q = 0; q < n_near; ++q) {
            const Cand& cd = cand_at(s.cand, wn[q]);
            const double4 a = fw.img_xyz[cd.id];
            const int atom = (int)(fw.img_id[cd.id] / (uint32_t)fw.imgs_per_atom);
            const double2 lj = fw.atom_lj64[atom];
            const double ax = a.x - o0, ay = a.y - o1, az = a.z - o2;
#pragma unroll
            for (int p = 0; p < Pol::kP; ++p) {
                const double dx = qx[p] - ax, dy = qy[p] - ay, dz = qz[p] - az;
                double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
                r2 = fmax(r2, cc.r2min);
                const double u = __drcp_rn(r2);
                const double u3 = u * u * u;
                nacc[p] = fma(u3, fma(lj.x, u3, -lj.y), nacc[p]);
            }
        }
    }
}

template <class Pol, int PREC>
__device__ void process_cta(EngineSmem& s, const Pol& pol, const FwDev& fw,
                            const CutoffConsts& cc) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;

    // 1. FP64 Cartesian points and the CTA box.
    double cx[Pol::kP], cy[Pol::kP], cz[Pol::kP];
    unsigned vmask = 0;
    double mn0 = INFINITY, mn1 = INFINITY, mn2 = INFINITY;
    double mx0 = -INFINITY, mx1 = -INFINITY, mx2 = -INFINITY;
#pragma unroll
    for (int p = 0; p < Pol::kP; ++p) {
        double f[3];
        const bool ok = pol.point(w, lane, p, f);
        frac_to_cart(fw.t, f[0], f[1], f[2], cx[p], cy[p], cz[p]);
        if (ok) {
            vmask |= 1u << p;
            mn0 = fmin(mn0, cx[p]); mn1 = fmin(mn1, cy[p]); mn2 = fmin(mn2, cz[p]);
            mx0 = fmax(mx0, cx[p]); mx1 = fmax(mx1, cy[p]); mx2 = fmax(mx2, cz[p]);
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
    const bool warp_live = __any_sync(0xffffffffu, vmask != 0);
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
    const double o0 = 0.5 * (lo0 + hi0), o1 = 0.5 * (lo1 + hi1), o2 = 0.5 * (lo2 + hi2);
    const int bul = borderline_ulps(
        cc.rc, cc.rc2f,
        sqrt((hi0 - lo0) * (hi0 - lo0) + (hi1 - lo1) * (hi1 - lo1) + (hi2 - lo2) * (hi2 - lo2)));

    // 2. local FP32 coordinates and the warp box
    float px[Pol::kP], py[Pol::kP], pz[Pol::kP], hi[Pol::kP], lo[Pol::kP];
    double nacc[PrecTraits<PREC>::near64 ? Pol::kP : 1];
#pragma unroll
    for (int p = 0; p < (PrecTraits<PREC>::near64 ? Pol::kP : 1); ++p) nacc[p] = 0.0;
    float wl0x = INFINITY, wl0y = INFINITY, wl0z = INFINITY;
    float wh0x = -INFINITY, wh0y = -INFINITY, wh0z = -INFINITY;
#pragma unroll
    for (int p = 0; p < Pol::kP; ++p) {
        px[p] = (float)(cx[p] - o0);
        py[p] = (float)(cy[p] - o1);
        pz[p] = (float)(cz[p] - o2);
        hi[p] = 0.f; lo[p] = 0.f;
        if (vmask & (1u << p)) {
            wl0x = fminf(wl0x, px[p]); wl0y = fminf(wl0y, py[p]); wl0z = fminf(wl0z, pz[p]);
            wh0x = fmaxf(wh0x, px[p]); wh0y = fmaxf(wh0y, py[p]); wh0z = fmaxf(wh0z, pz[p]);
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
            for (int cb = 0; cb < tot; cb += kThreads) {
                const int c = cb + tid;
                int pass = 0, g = 0;
                float4 cp = make_float4(0.f, 0.f, 0.f, 0.f);
                float nc6 = 0.f;
                if (c < tot) {
                    int a = 0, b = nr - 1;
                    while (a < b) {
                        const int mid = (a + b + 1) >> 1;
                        if (s.row_off[mid] <= c) a = mid; else b = mid - 1;
                    }
                    g = s.row_beg[a] + (c - s.row_off[a]);
                    const double4 ap = fw.img_xyz[g];
                    const float ax = (float)(ap.x - o0), ay = (float)(ap.y - o1),
                                az = (float)(ap.z - o2);
                    const float ddx = fmaxf(0.f, fmaxf(b0x - ax, ax - b1x));
                    const float ddy = fmaxf(0.f, fmaxf(b0y - ay, ay - b1y));
                    const float ddz = fmaxf(0.f, fmaxf(b0z - az, az - b1z));
                    pass = (ddx * ddx + ddy * ddy + ddz * ddz) < R2f;
                    if (pass) {
                        const float2 pr = fw.img_par[g];
                        cp = make_float4(ax, ay, az, pr.x);
                        nc6 = pr.y;
                    }
                }
                int npass;
                const int pos = block_exscan(pass, s.warp_tot, &npass);
                if (n_cand + npass > kMaxCand) {
                    __syncthreads();
                    warp_flush<Pol, PREC>(s, pol, fw, cc, n_cand, px, py, pz, hi, lo, nacc, wl0x,
                                          wl0y, wl0z, wh0x, wh0y, wh0z, warp_live, vmask, bul);
                    __syncthreads();
                    n_cand = 0;
                }
                if (pass) {
                    Cand& dst = s.cand[n_cand + pos];
                    dst.p = cp;
                    dst.nc6 = nc6;
                    dst.id = g;
                }
                n_cand += npass;
            }
            __syncthreads();
        }
    }
    if (n_cand > 0) {
        __syncthreads();
        warp_flush<Pol, PREC>(s, pol, fw, cc, n_cand, px, py, pz, hi, lo, nacc, wl0x, wl0y,
                              wl0z, wh0x, wh0y, wh0z, warp_live, vmask, bul);
    }
    // 4. store
#pragma unroll
    for (int p = 0; p < Pol::kP; ++p) {
        if (vmask & (1u << p)) {
            float e;
            if (PrecTraits<PREC>::near64)
                e = (float)(((double)hi[p] + (double)lo[p]) + nacc[PrecTraits<PREC>::near64 ? p : 0]);
            else
                e = PrecTraits<PREC>::comp ? __fadd_rn(hi[p], lo[p]) : hi[p];
            if (PREC != PREC_COUNT) e = fminf(e, kEnergyCap);
            pol.store(w, lane, p, e);
        }
    }
    __syncthreads();
}

}  // namespace er
