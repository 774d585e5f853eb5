// er_server.cu -- request server with continuous batching (er_server_*).
//
// One scheduler thread per server. A slot is a CUDA stream with its own
// Widom scratch; an admitted job's kernels go onto its slot's stream at once,
// so the device runs the kernels of every admitted job concurrently and new
// arrivals join while earlier ones are still running. Completion is detected
// with one event per slot. Frameworks (the image cell lists) and finished
// grids stay resident and are reused by later jobs.
//
// Admission. Every job's cost is estimated as points (grid points or
// insertions) x atom density, proportional to its pair terms. Jobs below a
// running median of the costs seen are "small". With two or more slots, half
// the slots are created at the device's highest stream priority and half at
// the lowest: the block scheduler then dispatches the CTAs of small jobs
// ahead of those of large ones (shortest-job-first at CTA granularity, with
// no preemption of running CTAs). The pending queue is scanned in arrival
// order (its first kScan jobs) and the first job with a free slot of its
// class is admitted (small jobs may use either class, large jobs only
// low-priority slots), unless the oldest job has waited longer than kAgeS:
// then nothing overtakes it and it takes any free slot. A job is admitted only when its device footprint fits
// the HBM budget after evicting unpinned cached grids (least recently used
// first). One slot is the plain one-job-at-a-time loop. The budget is
// reserved in the context's memory pool when the server is created.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "er_ctx.h"
#include "er_engine.cuh"
#include "er_nvtx.h"

namespace {

using Clock = std::chrono::steady_clock;
using GridKey = std::tuple<uint64_t, int, int, int>;

struct SrvFw {
    int fw_id = 0;
    size_t bytes = 0;
    uint64_t last_use = 0;
    int pins = 0;
};

struct SrvGrid {
    float* ptr = nullptr;
    size_t bytes = 0;  // the grid
    size_t cap = 0;    // its buffer (a recycled buffer may be larger)
    uint64_t last_use = 0;
    int pins = 0;
    bool ready = false;
};

struct SrvJob {
    er_job job{};
    er_job_status st{};
    int slot = -1;
    GridKey gkey{};
    double log_cost = 0.0;  // log of the admission cost estimate (set at submission)
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    er::HenryScratch hs;
    er::HenryOut* pinned = nullptr;  // host copy of the Widom reduction
    uint64_t ticket = 0;
    bool busy = false;
    bool high = false;               // created at the highest stream priority
};

constexpr double kAgeS = 0.05;       // a job waiting longer is overtaken by none
constexpr int kScan = 64;            // pending jobs examined per admission attempt

}  // namespace

struct er_server {
    er_ctx* ctx = nullptr;
    size_t budget = 0;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> pending;
    std::unordered_map<uint64_t, SrvJob> jobs;
    std::unordered_map<uint64_t, SrvFw> fws;
    std::map<GridKey, SrvGrid> grids;
    size_t bytes_fw = 0, bytes_grid = 0;
    uint64_t next_ticket = 1, tick = 0;
    bool stop = false;
    std::thread thr;
    Clock::time_point t0;
    double cost_log_ema = 0.0;   // running centre of log(cost)
    bool cost_seen = false;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    size_t scratch_bytes() const {
        size_t b = 0;
        for (const Slot& s : slots) b += s.hs.bytes();
        return b;
    }
    size_t used() const { return bytes_fw + bytes_grid + scratch_bytes(); }

    // Frees least recently used grids that no running job holds until
    // `need` more bytes fit the budget; returns whether they fit.
    bool make_room(size_t need, cudaStream_t st) {
        while (used() + need > budget) {
            auto victim = grids.end();
            for (auto it = grids.begin(); it != grids.end(); ++it)
                if (it->second.pins == 0 && it->second.ready &&
                    (victim == grids.end() || it->second.last_use < victim->second.last_use))
                    victim = it;
            if (victim == grids.end()) return false;
            cudaFreeAsync(victim->second.ptr, st);
            bytes_grid -= victim->second.cap;
            grids.erase(victim);
        }
        return true;
    }

    // With the budget full, a grid of `need` bytes takes over the buffer of the
    // least recently used idle grid whose buffer holds it with at most 25 %
    // to spare (failing that, at most 100 %), instead of freeing grids to the
    // pool and allocating: grid sizes vary continuously, and a pool whose
    // memory is cut into grids of other sizes must map new memory for the
    // request (measured stalls of up to 0.7 s on the request path). Returns
    // nullptr when no such grid exists.
    float* recycle(size_t need, size_t* cap) {
        if (used() + need <= budget) return nullptr;
        auto victim = grids.end();
        for (size_t spare : {need / 4, need}) {
            for (auto it = grids.begin(); it != grids.end(); ++it) {
                const SrvGrid& g = it->second;
                if (g.pins == 0 && g.ready && g.cap >= need && g.cap - need <= spare &&
                    (victim == grids.end() || g.last_use < victim->second.last_use))
                    victim = it;
            }
            if (victim != grids.end()) break;
        }
        if (victim == grids.end()) return nullptr;
        float* p = victim->second.ptr;
        *cap = victim->second.cap;
        bytes_grid -= victim->second.cap;
        grids.erase(victim);
        return p;
    }

    void finish(SrvJob& j, int status) {
        j.st.done = 1;
        j.st.status = status;
        j.st.finish_s = now();
    }

    // Points x atoms per A^3 (proportional to the pair terms of the job).
    double job_cost(const er_job& job) {
        double rho = 0.01;
        auto f = fws.find(job.fw_key);
        if (f != fws.end()) {
            const er::FwRecord* r = er::find_fw(ctx, f->second.fw_id);
            if (r && r->volume > 0) rho = r->n_atoms / r->volume;
        } else if (job.desc) {
            const double* t = job.desc->t_matrix;
            const double v = fabs(t[0] * (t[4] * t[8] - t[5] * t[7]) -
                                  t[1] * (t[3] * t[8] - t[5] * t[6]) +
                                  t[2] * (t[3] * t[7] - t[4] * t[6]));
            if (v > 0) rho = job.desc->n_atoms / v;
        }
        const double pts = job.kind == ER_JOB_GRID ? (double)job.nx * job.ny * job.nz
                                                   : (double)job.n_insertions;
        return std::max(pts, 1.0) * std::max(rho, 1e-4);
    }

    // A free slot for a job of the given class (-1: none).
    int pick_slot(bool small, bool any) const {
        int low = -1, high = -1;
        for (size_t i = 0; i < slots.size(); ++i) {
            if (slots[i].busy) continue;
            if (slots[i].high) {
                if (high < 0) high = (int)i;
            } else if (low < 0) {
                low = (int)i;
            }
        }
        if (slots.size() == 1 || any) return high >= 0 ? high : low;
        if (small) return high >= 0 ? high : low;
        return low;
    }

    // Admits (or resolves) one pending job; returns whether it did.
    bool admit_one() {
        if (pending.empty()) return false;
        bool any_free = false;
        for (const Slot& sl : slots) any_free |= !sl.busy;
        if (!any_free) return false;
        const double t_now = now();
        const bool aged = t_now - jobs[pending.front()].st.submit_s > kAgeS;
        int examined = 0;
        for (auto it = pending.begin(); it != pending.end() && examined < kScan;
             ++it, ++examined) {
            const uint64_t ticket = *it;
            SrvJob& j = jobs[ticket];
            const double lc = j.log_cost;
            if (!cost_seen) {
                cost_log_ema = lc;
                cost_seen = true;
            }
            const bool small = lc <= cost_log_ema;
            const bool head = it == pending.begin();
            const int slot = pick_slot(small, aged && head);
            if (slot < 0) {
                if (aged) return false;  // the aged head job goes first
                continue;
            }
            cost_log_ema += 0.05 * (lc - cost_log_ema);
            const int r = admit(ticket, j, slot);
            if (r == kWait) return false;
            pending.erase(it);
            if (r == kResolved) cv_done.notify_all();
            return true;
        }
        return false;
    }

    enum { kStarted = 0, kResolved = 1, kWait = 2 };

    // Starts job `ticket` on slot `slot_i`, or resolves it at once (a resident
    // grid, an error); kWait when its footprint does not fit while other jobs
    // run.
    int admit(uint64_t ticket, SrvJob& j, int slot_i) {
        Slot& sl = slots[slot_i];
        const er_job& job = j.job;
        ++tick;
        // a grid that is already resident completes at once
        if (job.kind == ER_JOB_GRID) {
            j.gkey = GridKey(job.fw_key, job.nx, job.ny, job.nz);
            auto g = grids.find(j.gkey);
            if (g != grids.end() && g->second.ready) {
                g->second.last_use = tick;
                j.st.grid_cache_hit = 1;
                j.st.start_s = now();
                if (job.grid_out_host)
                    cudaMemcpy(job.grid_out_host, g->second.ptr, g->second.bytes,
                               cudaMemcpyDeviceToHost);
                finish(j, ER_OK);
                return kResolved;
            }
        }
        // framework resident?
        auto f = fws.find(job.fw_key);
        if (f == fws.end()) {
            if (!job.desc) {
                finish(j, ER_ERR_NOT_FOUND);
                return kResolved;
            }
            int fw_id = 0;
            int st = er_framework_upload(ctx, job.desc, &fw_id);
            if (st != ER_OK) {
                finish(j, st);
                return kResolved;
            }
            SrvFw rec;
            rec.fw_id = fw_id;
            er_framework_bytes(ctx, fw_id, &rec.bytes);
            bytes_fw += rec.bytes;
            f = fws.emplace(job.fw_key, rec).first;
        }
        const er::FwRecord* fr = er::find_fw(ctx, f->second.fw_id);
        // footprint
        size_t need = 0;
        int64_t h_cap = 0;
        if (job.kind == ER_JOB_GRID) {
            need = (size_t)job.nx * job.ny * job.nz * sizeof(float);
        } else {
            // a slot's Widom scratch grows with headroom (to the next power
            // of two of insertions, at most 1.5x the job): a few growths per
            // slot, early, instead of one per larger job (each a pool
            // allocation that can stall once the pool's memory is cut into
            // grids)
            h_cap = (int64_t)1 << 20;
            while (h_cap < job.n_insertions) h_cap <<= 1;
            h_cap = std::max<int64_t>(job.n_insertions,
                                      std::min<int64_t>(h_cap, job.n_insertions + job.n_insertions / 2));
            const size_t want = (size_t)h_cap * 41 + (4u << 20);
            const size_t have = sl.hs.bytes();
            need = want > have ? want - have : 0;
        }
        size_t rcap = 0;
        float* rbuf = job.kind == ER_JOB_GRID ? recycle(need, &rcap) : nullptr;
        if (!rbuf && !make_room(need, sl.stream)) {
            // nothing left to evict: wait for running jobs, or fail if none run
            bool any_busy = false;
            for (const Slot& s : slots) any_busy |= s.busy;
            if (any_busy) return kWait;
            finish(j, ER_ERR_NOMEM);
            return kResolved;
        }
        f->second.last_use = tick;
        f->second.pins++;
        j.st.start_s = now();
        er::NvtxRange nvtx(job.kind == ER_JOB_GRID ? "server grid job launch"
                                                   : "server Henry job launch");
        int st = ER_OK;
        if (job.kind == ER_JOB_GRID) {
            SrvGrid g;
            g.bytes = need;
            g.cap = rbuf ? rcap : need;
            g.ptr = rbuf;
            if (!rbuf && cudaMallocFromPoolAsync((void**)&g.ptr, g.bytes, ctx->pool, sl.stream) !=
                             cudaSuccess) {
                cudaGetLastError();
                st = ER_ERR_NOMEM;
            } else {
                er::GridTask t;
                st = er::fill_grid_task(ctx, *fr, job.nx, job.ny, job.nz, g.ptr, t);
                if (st == ER_OK) st = er::launch_grid_plain_on(ctx, t, er::PREC_NEAR64, sl.stream);
                if (st == ER_OK && job.grid_out_host &&
                    cudaMemcpyAsync(job.grid_out_host, g.ptr, g.bytes, cudaMemcpyDeviceToHost,
                                    sl.stream) != cudaSuccess) {
                    cudaGetLastError();
                    st = ER_ERR_CUDA;
                }
                if (st == ER_OK) {
                    g.pins = 1;
                    g.last_use = tick;
                    bytes_grid += g.cap;
                    grids[j.gkey] = g;
                } else {
                    cudaFreeAsync(g.ptr, sl.stream);
                }
            }
        } else {
            st = er::henry_check(ctx, job.temperature, job.n_insertions, nullptr, 0, 0, 0);
            if (st == ER_OK) st = er::henry_reserve(ctx, sl.hs, h_cap, sl.stream);
            if (st == ER_OK)
                st = er::henry_enqueue(ctx, *fr, job.temperature, (int)job.n_insertions, job.seed,
                                       nullptr, 0, 0, 0, sl.stream, sl.hs, sl.pinned);
        }
        if (st != ER_OK) {
            f->second.pins--;
            finish(j, st);
            return kResolved;
        }
        cudaEventRecord(sl.done, sl.stream);
        sl.busy = true;
        sl.ticket = ticket;
        j.slot = slot_i;
        return kStarted;
    }

    bool reap() {
        bool any = false;
        for (Slot& sl : slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            SrvJob& j = jobs[sl.ticket];
            int status = ER_OK;
            if (q != cudaSuccess) {
                cudaGetLastError();
                status = ER_ERR_CUDA;
            }
            // a bounded wait that gave up in some kernel of the context since the
            // last check: the job finishing now is failed (the word is per
            // context, so a concurrent job's fault may land on this one)
            if (status == ER_OK && er::take_fault(ctx) != ER_OK) status = ER_ERR_CUDA;
            if (j.job.kind == ER_JOB_HENRY && status == ER_OK)
                er::henry_finish(*sl.pinned, j.job.n_insertions, j.job.temperature, &j.st.henry);
            if (j.job.kind == ER_JOB_GRID) {
                auto g = grids.find(j.gkey);
                if (g != grids.end()) {
                    g->second.pins--;
                    g->second.ready = status == ER_OK;
                }
            }
            auto f = fws.find(j.job.fw_key);
            if (f != fws.end()) f->second.pins--;
            finish(j, status);
            sl.busy = false;
            any = true;
        }
        if (any) cv_done.notify_all();
        return any;
    }

    void run() {
        cudaSetDevice(ctx->device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            bool progress = reap();
            while (!stop && admit_one()) progress = true;
            bool busy = false;
            for (const Slot& s : slots) busy |= s.busy;
            if (stop && !busy) break;
            if (!progress) cv_work.wait_for(lk, std::chrono::microseconds(busy ? 20 : 2000));
        }
    }
};

using namespace er;

extern "C" {

int er_server_create(er_ctx* ctx, size_t hbm_budget_bytes, int slots, er_server** out) {
    if (!ctx || !out || slots < 1 || slots > 64 || hbm_budget_bytes == 0) return ER_ERR_INVALID;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    er_server* s = new er_server();
    s->ctx = ctx;
    s->budget = hbm_budget_bytes;
    s->t0 = Clock::now();
    s->slots.resize(slots);
    int prio_least = 0, prio_greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess) {
        cudaGetLastError();
        prio_least = prio_greatest = 0;
    }
    for (int i = 0; i < slots; ++i) {
        Slot& sl = s->slots[i];
        sl.high = slots > 1 && i < slots / 2;
        const int prio = slots == 1 ? 0 : (sl.high ? prio_greatest : prio_least);
        if (cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost((void**)&sl.pinned, sizeof(HenryOut)) != cudaSuccess) {
            cudaGetLastError();
            er_server_destroy(s);
            return set_error(ctx, ER_ERR_CUDA, "server: stream/event creation failed");
        }
    }
    // Reserve the budget in the context's pool up front (allocate, free: the
    // pool keeps the memory), so that admissions carve grids and scratch out
    // of mapped memory instead of growing the pool on the request path.
    {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            free_b = 0;
        }
        size_t want = std::min(hbm_budget_bytes, (size_t)(0.9 * (double)free_b));
        void* p = nullptr;
        while (want >= (64u << 20)) {
            if (cudaMallocFromPoolAsync(&p, want, ctx->pool, ctx->stream) == cudaSuccess) {
                cudaFreeAsync(p, ctx->stream);
                break;
            }
            cudaGetLastError();
            want /= 2;
        }
        cudaStreamSynchronize(ctx->stream);
    }
    // Each slot's Widom scratch is reserved now as well (an eighth of the
    // budget over all slots, at most 2^24 insertions per slot; counted in the
    // budget): Henry jobs up to that size never grow it on the request path,
    // where the pool's memory may already be cut up by grids.
    {
        const int64_t fit = (int64_t)(hbm_budget_bytes / 8 / (size_t)slots / 41);
        int64_t cap = 0;
        for (int64_t c = (int64_t)1 << 16; c <= std::min<int64_t>(fit, (int64_t)1 << 24); c <<= 1)
            cap = c;
        if (cap > 0)
            for (Slot& sl : s->slots)
                if (er::henry_reserve(ctx, sl.hs, cap, sl.stream) != ER_OK) break;
        for (Slot& sl : s->slots) cudaStreamSynchronize(sl.stream);
    }
    s->thr = std::thread([s]() { s->run(); });
    *out = s;
    return ER_OK;
}

int er_server_submit(er_server* s, const er_job* job, uint64_t* ticket) {
    if (!s || !job || !ticket) return ER_ERR_INVALID;
    if (job->kind != ER_JOB_GRID && job->kind != ER_JOB_HENRY) return ER_ERR_INVALID;
    if (job->kind == ER_JOB_GRID && (job->nx < 2 || job->ny < 2 || job->nz < 2))
        return ER_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return ER_ERR_INVALID;
    const uint64_t t = s->next_ticket++;
    SrvJob j;
    j.job = *job;
    j.st.submit_s = s->now();
    j.log_cost = log(s->job_cost(*job));
    s->jobs.emplace(t, j);
    s->pending.push_back(t);
    *ticket = t;
    s->cv_work.notify_one();
    return ER_OK;
}

int er_server_poll(er_server* s, uint64_t ticket, er_job_status* st) {
    if (!s || !st) return ER_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return ER_ERR_NOT_FOUND;
    *st = it->second.st;
    return ER_OK;
}

int er_server_wait(er_server* s, uint64_t ticket, double timeout_s, er_job_status* st) {
    if (!s || !st || !(timeout_s >= 0)) return ER_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return ER_ERR_NOT_FOUND;
    const auto until = Clock::now() + std::chrono::duration<double>(timeout_s);
    while (!s->jobs[ticket].st.done) {
        if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout &&
            !s->jobs[ticket].st.done) {
            *st = s->jobs[ticket].st;
            return ER_ERR_TIMEOUT;
        }
    }
    *st = s->jobs[ticket].st;
    return ER_OK;
}

int er_server_grid(er_server* s, uint64_t ticket, const float** grid) {
    if (!s || !grid) return ER_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end() || it->second.job.kind != ER_JOB_GRID || !it->second.st.done)
        return ER_ERR_NOT_FOUND;
    auto g = s->grids.find(it->second.gkey);
    if (g == s->grids.end() || !g->second.ready) return ER_ERR_NOT_FOUND;
    *grid = g->second.ptr;
    return ER_OK;
}

double er_server_now(const er_server* s) { return s ? s->now() : 0.0; }

int er_server_bytes(const er_server* s, size_t* bytes) {
    if (!s || !bytes) return ER_ERR_INVALID;
    std::lock_guard<std::mutex> lk(const_cast<er_server*>(s)->mu);
    *bytes = s->used();
    return ER_OK;
}

void er_server_destroy(er_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (uint64_t t : s->pending) s->finish(s->jobs[t], ER_ERR_INVALID);
        s->pending.clear();
        s->cv_work.notify_all();
        s->cv_done.notify_all();
    }
    if (s->thr.joinable()) s->thr.join();
    cudaSetDevice(s->ctx->device);
    for (Slot& sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        sl.hs.release();
        if (sl.pinned) cudaFreeHost(sl.pinned);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    for (auto& kv : s->grids) cudaFreeAsync(kv.second.ptr, s->ctx->stream);
    cudaStreamSynchronize(s->ctx->stream);
    for (auto& kv : s->fws) er_framework_release(s->ctx, kv.second.fw_id);
    for (Slot& sl : s->slots)
        if (sl.stream) cudaStreamDestroy(sl.stream);
    delete s;
}

}  // extern "C"
