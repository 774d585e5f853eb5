"""Benchmark of the LJ grid hot path on the 256-framework batch workload.

Workload (one "step"): grids of 256 seeded triclinic frameworks (a, b, c in
[8, 40] A, angles in [60, 120] deg, 100-5000 atoms log-uniform capped at 0.16
atoms/A^3, 8 atom types, probes CH4 / Xe / Kr, grid spacing 0.1-0.2 A, cutoff
12.5 A) computed by one persistent launch over a device work queue replayed
as a CUDA graph, in the default precision mode (ER_PREC_NEAR64: FP32 pair
terms, pairs of atoms within 5 A of a warp's points in FP64; within 1e-5
relative of FP64 on E < -10 K points). Data are synthetic (no dataset ships
with the reference).

value    pair terms/s of the batched launch, inputs resident, device-timed with
         CUDA events on the library's stream (in-cutoff pair terms counted
         exactly by the same traversal in counting mode, outside the timing)
e2e      the same metric through the C ABI with host buffers: per step every
         framework is uploaded (host preparation + H2D), the batch runs, and
         every grid is copied back to pinned host memory
roofline pair terms/s x 11 FP32-pipe instructions per pair against the
         device's FP32 FMA issue rate measured by er_probe_fp32_rate
errors   the batch grids and the Widom K_H against the FP64 oracle: sampled
         points of every grid, K_H of four Widom frameworks at full size
cpu_baseline the reference's own ComputeGridSheet (oracle/_ref) on a bounded
         sample of the same grids and of Widom insertion points, all host cores

`--impl reference` times only the reference's CPU implementation (on
frameworks built by oracle/workloads.py, without this library).
Multi-GPU (torchrun): every rank runs its own 256-framework batch (weak
scaling, no collective on the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LJ pair terms/s & Widom insertions/s; served p50/p99 vs plain, same B200"
PAIR_INSTR = 11  # FP32-pipe instructions credited per in-cutoff pair term
WORKLOAD = "256-framework batched LJ grids (config 2)"
DEEP = -10.0     # K: below this the grid tolerance is 1e-5 relative


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(v, pg):
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v, pg):
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"er_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(rank, n=256):
    from emptyroom_b200 import synth
    return synth.config2(n_frameworks=n, seed=1000 + 100000 * rank)


def upload_all(ctx, fws):
    return ctx.upload_many([(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws])


def count_pairs(ctx, ups, dims_list):
    """Exact in-cutoff pair terms per job (counting traversal)."""
    import torch
    counts = []
    for u, dims in zip(ups, dims_list):
        buf = torch.empty(dims, dtype=torch.float32, device="cuda")
        ctx.count_pairs_device(u, dims, buf.data_ptr())
        ctx.synchronize()
        counts.append(int(buf.double().sum().item()))
        del buf
    return counts


def flush_l2(buf):
    buf.fill_(1.0)


def time_plan(ctx, plan, steps, warmup, l2buf):
    import torch
    s = torch.cuda.ExternalStream(ctx.stream_ptr)
    for _ in range(warmup):
        plan.run()
    ctx.synchronize()
    times = []
    for _ in range(steps):
        flush_l2(l2buf)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        plan.run()
        e1.record(s)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    return times


def ref_grid_sample(fws, target_s, rng, cores, chunk=256):
    """The reference's ComputeGridSheet (oracle/_ref; the oracle's image loop
    when the reference was not built here), called on one-point axes, at
    random grid points of frameworks drawn by grid size until target_s seconds
    of work: (pair terms, seconds, samples). Each point costs the reference
    what it costs inside a whole sheet (every image of every atom); the pair
    terms of the sample are counted by the cell-list oracle."""
    import oracle
    use_ref = oracle.ref_available()
    pairs = secs = 0.0
    sample = []
    # frameworks drawn in proportion to their grid points: the sample's pair
    # terms per second then estimate the whole batch's, whose frameworks cost
    # the reference anything from a few hundred to ~1e6 image evaluations per point
    w = np.array([float(np.prod(f.dims)) for f in fws])
    w /= w.sum()
    while secs < target_s:
        k = int(rng.choice(len(fws), p=w))
        f = fws[k]
        P = f.particles()
        dims = np.array(f.dims)
        pts = rng.integers(0, dims, size=(chunk, 3)) / (dims - 1.0)
        t0 = time.perf_counter()
        if use_ref:
            oracle.ref_points(P, f.t_matrix, f.rep, f.rc2, pts, n_threads=cores)
        else:
            oracle.points(P, f.t_matrix, f.rep, f.rc2, pts, n_threads=cores)
        secs += time.perf_counter() - t0
        pairs += float(oracle.points_cells(P, f.t_matrix, f.rep, f.rc2, pts,
                                           n_threads=cores)[2].sum())
        sample.append(f"fw{k}")
    return pairs, secs, sample


def ref_widom_sample(f, target_s, cores, seed=0):
    """The reference's LJ routine (ComputeGridSheet at one-point axes, the sum
    of src/doHenry.h:70-98) at the first Philox insertion points of stream
    `seed`, plus exp(-E/T) accumulation, until target_s seconds: (insertions,
    pair terms, seconds)."""
    import oracle
    use_ref = oracle.ref_available()
    P = f.particles()
    n_done = 0
    pairs = secs = 0.0
    chunk = 2048
    while secs < target_s:
        pts = oracle.insertion_points(seed, chunk, n_done)
        t0 = time.perf_counter()
        if use_ref:
            e = oracle.ref_points(P, f.t_matrix, f.rep, f.rc2, pts, n_threads=cores)
        else:
            e = oracle.points(P, f.t_matrix, f.rep, f.rc2, pts, 1e-16, n_threads=cores)
        np.exp(-e / 298.0).sum()
        secs += time.perf_counter() - t0
        pairs += float(oracle.points_cells(P, f.t_matrix, f.rep, f.rc2, pts, 1e-16,
                                           n_threads=cores)[2].sum())
        n_done += chunk
        chunk = min(chunk * 2, 65536)
    return n_done, pairs, secs


def cpu_baseline(fws, fw_widom, target_s=10.0):
    """The reference's own CPU code (oracle/_ref) on all host cores: whole
    x-sheets of the batch's grids, and Widom insertion points of a config-4
    framework; each leg a bounded sample extrapolated per pair term."""
    import oracle
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(7)
    pairs, secs, sample = ref_grid_sample(fws, target_s, rng, cores)
    n_ins, wpairs, wsecs = ref_widom_sample(fw_widom, target_s * 0.6, cores)
    return {"value": pairs / secs, "unit": "pair-terms/s", "cores": cores,
            "kind": "reference" if oracle.ref_available() else "port",
            "sample": f"{len(sample)} draws of 256 random grid points each, the framework of "
                      f"each draw picked in proportion to its grid size ({len(set(sample))} "
                      f"distinct of the {len(fws)} batch frameworks; {pairs:.3g} pair terms "
                      f"in {secs:.1f} s)",
            "widom": {"insertions_per_s": n_ins / wsecs, "pair_terms_per_s": wpairs / wsecs,
                      "sample": f"first {n_ins} Philox insertions of a config-4 cell (Xe) "
                                f"in {wsecs:.1f} s, extrapolated per insertion"}}


def grid_errors_block(fws, outs, cores, seed=11, n_deep=192, n_shallow=32, n_uniform=64):
    """Error of every batch grid against the FP64 oracle (cell-list form) on
    sampled points: up to n_deep points with E < -10 K, n_shallow with
    -10 K <= E < 0 and n_uniform anywhere, chosen from the GPU grid."""
    import torch

    import oracle
    rng = np.random.default_rng(seed)
    deep_max, deep_p99, n_deep_pts = [], [], []
    all_deep_rel, shallow_ratio, pos_rel = [], [], []
    cap_ok = True
    for f, o in zip(fws, outs):
        flat = o.reshape(-1)
        picks = []
        for sel, cnt in ((flat < DEEP, n_deep), ((flat >= DEEP) & (flat < 0), n_shallow)):
            idx = torch.nonzero(sel).reshape(-1)
            if idx.numel():
                take = torch.from_numpy(rng.choice(idx.numel(), size=min(cnt, idx.numel()),
                                                   replace=False)).to(idx.device)
                picks.append(idx[take].cpu().numpy())
        picks.append(rng.integers(0, flat.numel(), size=n_uniform))
        idx = np.unique(np.concatenate(picks))
        got = flat[torch.from_numpy(idx).to(flat.device)].double().cpu().numpy()
        dims = np.array(f.dims)
        ijk = np.stack(np.unravel_index(idx, f.dims), -1)
        pts = ijk / (dims - 1.0)
        ref, S, _ = oracle.points_cells(f.particles(), f.t_matrix, f.rep, f.rc2, pts, 1e-12,
                                        n_threads=cores)
        d = np.abs(got - ref)
        deep = ref < DEEP
        shallow = (ref >= DEEP) & (ref < 0)
        pos = (ref >= 0) & (ref < 1e10)
        rel = d[deep] / np.abs(ref[deep])
        n_deep_pts.append(int(deep.sum()))
        deep_max.append(float(rel.max()) if rel.size else None)
        deep_p99.append(float(np.percentile(rel, 99)) if rel.size else None)
        all_deep_rel.append(rel)
        if shallow.any():  # |dE| against 1e-5 |E| + 2e-6 S, the bound of the tests
            shallow_ratio.append(float((d[shallow] / (1e-5 * np.abs(ref[shallow]) +
                                                      2e-6 * S[shallow])).max()))
        if pos.any():
            pos_rel.append(float((d[pos] / np.maximum(np.abs(ref[pos]), 1.0)).max()))
        cap = ref >= 1e30
        cap_ok &= bool(np.all(got[cap] == np.float32(1e30)))
    rel = np.concatenate(all_deep_rel)
    return {"workload": f"all {len(fws)} batch grids (default mode), points sampled from each "
                        f"grid: <= {n_deep} with E < {DEEP:g} K, <= {n_shallow} with "
                        f"{DEEP:g} K <= E < 0, {n_uniform} uniform; FP64 oracle (cell-list "
                        f"sum of the reference's terms)",
            "deep": {"points": int(rel.size), "max_rel": float(rel.max()),
                     "p99_rel": float(np.percentile(rel, 99)),
                     "n_over_1e-5": int((rel > 1e-5).sum()),
                     "grids_with_points": int(sum(1 for n in n_deep_pts if n))},
            "shallow_max_over_bound": max(shallow_ratio) if shallow_ratio else None,
            "pos_max_rel": max(pos_rel) if pos_rel else None,
            "cap_ok": cap_ok,
            "per_grid_deep_max_rel": [None if v is None else float(f"{v:.3g}")
                                      for v in deep_max],
            "per_grid_deep_p99_rel": [None if v is None else float(f"{v:.3g}")
                                      for v in deep_p99],
            "per_grid_deep_points": n_deep_pts}


def run_ours(args, ws, rank, local, pg):
    import torch

    import emptyroom_b200 as er
    torch.cuda.set_device(local)
    ctx = er.Context(local)
    fws = make_workload(rank, args.frameworks)
    ups = upload_all(ctx, fws)
    counts = count_pairs(ctx, ups, [f.dims for f in fws])
    pairs_step = float(sum(counts))
    points_step = float(sum(int(np.prod(f.dims)) for f in fws))
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    jobs = [(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)]
    # one persistent launch in the default (NEAR64) mode; the kernel variant of
    # each job class picked by the autotuner at plan creation, outside the timing
    plan = ctx.batch_plan(jobs, er.ER_BATCH_PERSISTENT | er.ER_BATCH_AUTOTUNE)
    tiles = [plan.tile(k) for k in range(len(jobs))]
    l2buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    fp32_rate = ctx.fp32_rate(0.2)

    barrier(pg)
    clocks = ClockSampler(local)
    clocks.start()
    times = time_plan(ctx, plan, args.steps, args.warmup, l2buf)
    clk = clocks.stop()
    barrier(pg)
    t_step = max_over_ranks(sum(times) / len(times), pg)
    total_pairs = sum_over_ranks(pairs_step, pg)
    value = total_pairs / t_step

    # the all-FP32 form: every pair term in FP32 (ER_PREC_COMP)
    comp = ctx.batch_plan(jobs, er.ER_BATCH_PERSISTENT | er.ER_BATCH_AUTOTUNE |
                          er.ER_BATCH_COMP)
    ctimes = time_plan(ctx, comp, max(2, args.steps // 2), 1, l2buf)
    t_comp = max_over_ranks(sum(ctimes) / len(ctimes), pg)
    comp.close()

    # plain per-framework launches (same grids, one launch per framework, graph-replayed)
    plain = ctx.batch_plan(jobs, er.ER_BATCH_PLAIN | er.ER_BATCH_AUTOTUNE)
    ptimes = time_plan(ctx, plain, max(2, args.steps // 2), 1, l2buf)
    t_plain = max_over_ranks(sum(ptimes) / len(ptimes), pg)
    plain_value = total_pairs / t_plain
    plain_launches = plain.launches
    plain.close()
    plan.run()  # outs hold the default-mode grids for the error check below
    ctx.synchronize()

    # e2e through the C ABI with host buffers
    ref_outs = [o.cpu().numpy().copy() for o in outs[:2]]
    host = torch.empty(int(points_step), dtype=torch.float32, pin_memory=True)
    offs = np.cumsum([0] + [int(np.prod(f.dims)) for f in fws])
    for u in ups:
        u.release()
    plan.close()
    e2e_times = []
    h2d = d2h = 0
    # host inputs: the mixed particle arrays of every framework (what the
    # reference's loaders produce); the timed calls upload and grid them
    host_items = [(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws]
    for step in range(args.warmup + args.steps):
        barrier(pg)
        t0 = time.perf_counter()
        ups2 = ctx.upload_many(host_items)
        host_jobs = [(u, f.dims, host.data_ptr() + 4 * int(offs[k]))
                     for k, (u, f) in enumerate(zip(ups2, fws))]
        ctx.grid_batch(host_jobs, er.ER_BATCH_PERSISTENT | er.ER_BATCH_HOST_OUT |
                       er.ER_BATCH_AUTOTUNE)
        dt = time.perf_counter() - t0
        if step == 0:
            # what er_framework_upload_many copies up: per atom its FP64
            # position and sig2 (32 B), FP64 (C12, C6) (16 B) and FP32
            # (C12, -C6) (8 B); per framework a 240-byte build record (copied
            # before each of the two build passes) and a block offset (the
            # image cell lists are built on the device)
            h2d = sum(56 * len(it[0]) + 484 for it in host_items) + 4
            d2h = int(points_step) * 4
            hv = host.numpy()
            for k in range(2):
                assert np.array_equal(hv[offs[k]:offs[k + 1]].reshape(fws[k].dims), ref_outs[k])
        for u in ups2:
            u.release()
        if step >= args.warmup:
            e2e_times.append(dt)
    t_e2e = max_over_ranks(sum(e2e_times) / len(e2e_times), pg)

    # roofline of the dominant (persistent) kernel
    t_kernel = sum(times) / len(times)
    achieved = pairs_step * PAIR_INSTR / t_kernel
    roof = {"bound": "fp32", "achieved": achieved / 1e12, "peak": fp32_rate / 1e12,
            "unit": "Tinst/s", "frac": achieved / fp32_rate,
            "peak_source": "measured FP32 FFMA issue rate (er_probe_fp32_rate) on this GPU",
            "traffic": load_traffic(points_step)}
    # the grid store against the measured HBM copy bandwidth (not the bound)
    roof["grid_store_gbs"] = 4.0 * points_step / t_kernel / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        hbm = json.load(open(peaks_path)).get("hbm_gbs")
        if hbm:
            roof["hbm_peak_gbs"] = hbm
            roof["grid_store_frac_of_measured_hbm"] = roof["grid_store_gbs"] / hbm
    line = {
        "metric": METRIC, "value": value, "unit": "pair-terms/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded frameworks; no dataset ships with the reference)",
        "config": {"workload": WORKLOAD,
                   "frameworks": len(fws), "precision": "ER_PREC_NEAR64 (default)",
                   "grid_points_per_step": int(points_step), "pair_terms_per_step": int(pairs_step),
                   "cutoff_A": 12.5, "spacing_A": [0.1, 0.2],
                   "l2": "flushed between timed steps (256 MB write)",
                   "tile_p8_jobs": int(sum(1 for t in tiles if t == 8)),
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
        "e2e": {"value": total_pairs / t_e2e, "unit": "pair-terms/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": t_e2e * 1e3},
        "gpu_launches": args.steps * 1,
        "roofline": roof,
        "clocks": clk,
        "plain": {"value": plain_value, "unit": "pair-terms/s", "launches_per_step": plain_launches,
                  "batched_over_plain": value / plain_value},
        "comp": {"value": total_pairs / t_comp, "unit": "pair-terms/s",
                 "ms_per_step": t_comp * 1e3, "roofline_frac":
                     pairs_step * PAIR_INSTR / (sum(ctimes) / len(ctimes)) / fp32_rate,
                 "note": "same batch with every pair term in FP32 (ER_PREC_COMP): faster, "
                         "but outside 1e-5 relative on some E < 0 points"},
    }
    # the FP64 reciprocal seed the default mode's near pairs refine by one
    # Newton step (their error is its square)
    line["rcp64_seed_max_rel_err"] = ctx.rcp64_seed_error()
    cores = os.cpu_count() or 1
    if rank == 0 and ws == 1 and not args.no_errors:
        line["errors"] = {"grids": grid_errors_block(fws, outs, cores)}
    del outs
    # the Widom and serving forms of the metric, at N = 1 (the batch above is
    # the scaled workload)
    if ws == 1:
        line["config1"] = run_config1(ctx)
        line["extras"] = run_extras(ctx)
        line["batch_small"] = run_batch_small(ctx, fws, l2buf, fp32_rate)
    if ws == 1 and not args.no_widom:
        line["widom"] = run_widom(ctx, args, fp32_rate, errors=not args.no_errors)
        if "kh_errors" in line["widom"]:
            line.setdefault("errors", {})["kh"] = line["widom"].pop("kh_errors")
    if ws == 1 and not args.no_serving:
        line["serving"] = run_serving(ctx, args)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from emptyroom_b200 import synth
        line["cpu_baseline"] = cpu_baseline(fws, synth.config4(1)[0])
        line["cpu_baseline"]["config1_grid_s"] = cpu_config1_grid()
        line["cpu_baseline"]["pockets_129cube_s"] = cpu_pockets_ref()
    ctx.close()
    return line


def run_batch_small(ctx, fws, l2buf, fp32_rate, dims=(32, 32, 32)):
    """Many small jobs, where one launch per job leaves the GPU idle: the 256
    batch frameworks each on a 32^3 grid (the config-1 grid size: 16-32
    bricks per job against 444 resident CTA slots), one persistent launch
    against one plain launch per job (both graph-replayed, default mode)."""
    import torch

    import emptyroom_b200 as er
    ups = upload_all(ctx, fws)
    pairs = float(sum(count_pairs(ctx, ups, [dims] * len(fws))))
    outs = [torch.empty(dims, dtype=torch.float32, device="cuda") for _ in fws]
    jobs = [(u, dims, o.data_ptr()) for u, o in zip(ups, outs)]
    res = {"workload": f"{len(fws)} batch frameworks, each on a {dims[0]}^3 grid",
           "pair_terms_per_step": int(pairs)}
    for name, mode in (("persistent", er.ER_BATCH_PERSISTENT), ("plain", er.ER_BATCH_PLAIN)):
        plan = ctx.batch_plan(jobs, mode | er.ER_BATCH_AUTOTUNE)
        ts = time_plan(ctx, plan, 10, 3, l2buf)
        t = sum(ts) / len(ts)
        res[name] = {"ms_per_step": t * 1e3, "pair_terms_per_s": pairs / t,
                     "launches_per_step": plan.launches,
                     "roofline_frac": pairs * PAIR_INSTR / t / fp32_rate}
        plan.close()
    res["persistent_over_plain"] = res["persistent"]["pair_terms_per_s"] / \
        res["plain"]["pair_terms_per_s"]
    for u in ups:
        u.release()
    return res


def run_widom(ctx, args, fp32_rate, errors=True):
    """Widom batch (config 4): per framework the 0.2 A grid, its pocket mask by
    GPU connected-components labelling, then er_henry with that device mask;
    64 frameworks x 1e7 insertions, Xe at 298 K. Timed through er_henry_batch
    (concurrent pipelines) and, beside it, as the sequence of single calls."""
    import torch

    from emptyroom_b200 import synth
    T = 298.0
    fws = synth.config4(args.widom_frameworks)
    ups = ctx.upload_many([(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws])
    dims = fws[0].dims
    g = torch.empty(dims, dtype=torch.float32, device="cuda")
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    cnt = torch.empty(dims, dtype=torch.float32, device="cuda")
    n_ins = int(args.insertions)
    s = torch.cuda.ExternalStream(ctx.stream_ptr)

    def one(k, u):
        ctx.grid_device(u, dims, g.data_ptr())
        n_p = ctx.block_pockets_device(g.data_ptr(), dims, T, m.data_ptr())
        r = ctx.henry_device_mask(u, T, n_ins, k, m.data_ptr(), dims)
        return n_p, r

    seeds = list(range(len(ups)))
    one(0, ups[0])  # warm-up
    ctx.henry_batch(ups[:3], T, n_ins, seeds[:3], block_dims=dims)
    ctx.synchronize()
    # the sequence of single calls (one stream, host round trips in between)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    seq = [one(k, u) for k, u in enumerate(ups)]
    e1.record(s)
    e1.synchronize()
    seq_s = e0.elapsed_time(e1) * 1e-3  # device-timed: all of it is on the context's stream
    # er_henry_batch: its pipelines run on their own streams, so the step is
    # timed on the host around the call (it returns when every result is in)
    ctx.synchronize()
    t0 = time.perf_counter()
    kh, npk = ctx.henry_batch(ups, T, n_ins, seeds, block_dims=dims)
    dev = time.perf_counter() - t0
    res = list(zip(npk, kh))
    assert [r[1] for r in res] == [r[1] for r in seq]  # bit for bit
    # pair terms: exact for the grids; for the insertions the grid's mean
    # in-cutoff pairs per point (insertions are uniform in the cell)
    grid_pairs = ins_pairs = 0.0
    mean_pairs = []
    for u in ups:
        ctx.count_pairs_device(u, dims, cnt.data_ptr())
        ctx.synchronize()
        c = float(cnt.double().sum().item())
        grid_pairs += c
        mean_pairs.append(c / float(np.prod(dims)))
        ins_pairs += mean_pairs[-1] * n_ins
    # the Widom pipeline of one framework alone (Philox points, bin layout,
    # energy kernel, FP64 log-sum-exp), device-timed on the library's stream,
    # with the energy kernel's own time from the library's stage events
    ctx.grid_device(ups[0], dims, g.data_ptr())
    ctx.block_pockets_device(g.data_ptr(), dims, T, m.data_ptr())
    ctx.set_timing(True)
    ts, stages = [], []
    for k in range(6):
        e0.record(s)
        ctx.henry_device_mask(ups[0], T, n_ins, 0, m.data_ptr(), dims)
        e1.record(s)
        e1.synchronize()
        if k:
            ts.append(e0.elapsed_time(e1) * 1e-3)
            stages.append(ctx.henry_timing())
    ctx.set_timing(False)
    t_pipe = sum(ts) / len(ts)
    t_energy = sum(st["energy_ms"] for st in stages) / len(stages) * 1e-3
    stage_ms = {k: sum(st[k] for st in stages) / len(stages) for k in stages[0]}
    unblocked = n_ins - seq[0][1]["n_blocked"]
    pipe_pairs = mean_pairs[0] * unblocked
    total_ins = n_ins * len(fws)
    out = {"workload": f"{len(fws)} config-1 cells, Xe 298 K: 0.2 A grid {list(dims)} -> "
                       f"GPU pocket mask -> {n_ins:.0e} Philox insertions each (config 4)",
           "insertions_per_s": total_ins / dev, "unit": "insertions/s",
           "ms_per_step": dev * 1e3,
           "timing": "host clock around er_henry_batch (synchronised before; the call "
                     "returns when all results are on the host)",
           "sequential_single_calls": {"ms_per_step": seq_s * 1e3,
                                       "insertions_per_s": total_ins / seq_s},
           "pair_terms_per_s": (grid_pairs + ins_pairs) / dev,
           "pair_terms_note": "grid pairs exact; insertion pairs = insertions x grid mean",
           "n_pockets_total": int(sum(r[0] for r in res)),
           "n_blocked_total": int(sum(r[1]["n_blocked"] for r in res)),
           "roofline": {"bound": "fp32", "unit": "Tinst/s", "peak": fp32_rate / 1e12,
                        "kernel": "henry_energy_kernel",
                        "achieved": pipe_pairs * PAIR_INSTR / t_energy / 1e12,
                        "frac": pipe_pairs * PAIR_INSTR / t_energy / fp32_rate,
                        "pair_terms_per_launch": pipe_pairs,
                        "energy_kernel_ms_per_1e7": t_energy * 1e3 * 1e7 / n_ins,
                        "pipeline_ms_per_1e7": t_pipe * 1e3 * 1e7 / n_ins,
                        "pipeline_frac": pipe_pairs * PAIR_INSTR / t_pipe / fp32_rate,
                        "stage_ms": stage_ms,
                        "note": "one framework's Widom pipeline on the library's stream; "
                                "the energy kernel timed by the library's stage events "
                                "(er_henry_last_timing), the pipeline by CUDA events around "
                                "the call; pair terms = unblocked insertions x the 0.2 A "
                                "grid's mean in-cutoff pairs per point"}}
    if errors:
        out["kh_errors"] = kh_errors(ctx, fws, ups, res, T, n_ins, dims)
    for u in ups:
        u.release()
    return out


def kh_errors(ctx, fws, ups, res, T, n_ins, dims, picks=(0, 21, 42, 63)):
    """K_H of four config-4 frameworks at the full insertion count, from the
    timed er_henry_batch, against the FP64 oracle: the oracle's own 0.2 A grid
    and pocket blocking (the reference's flood fill restated), the same Philox
    points, the cell-list sum of the reference's terms."""
    import torch

    import oracle
    cores = os.cpu_count() or 1
    out = {"workload": f"config-4 frameworks {list(picks)}, {n_ins:.0e} insertions each, "
                       "Xe 298 K, pockets masked"}
    rows = []
    g = torch.empty(dims, dtype=torch.float32, device="cuda")
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    for k in picks:
        if k >= len(fws):
            continue
        f = fws[k]
        P = f.particles()
        ctx.grid_device(ups[k], dims, g.data_ptr())
        ctx.block_pockets_device(g.data_ptr(), dims, T, m.data_ptr())
        ctx.synchronize()
        mask_gpu = m.cpu().numpy()
        t0 = time.perf_counter()
        E = oracle.grid_cells(P, f.t_matrix, f.rep, f.rc2, dims, n_threads=cores)
        blocked, n_p, _ = oracle.block_pockets(E, T)
        mask_o = ((blocked == 1e13) & (E != 1e13)).astype(np.uint8)
        o = oracle.henry_cells(P, f.t_matrix, f.rep, f.rc2, T, k, n_ins, mask=mask_o,
                               n_threads=cores)
        kh_o = o["sum_w"] / n_ins / T / 8.314
        kh = res[k][1]["kh_mol_m3_pa"]
        rows.append({"fw": k, "kh_rel_err": abs(kh - kh_o) / kh_o, "kh_gpu": kh,
                     "kh_oracle": kh_o, "mask_equal": bool(np.array_equal(mask_gpu, mask_o)),
                     "n_pockets": [res[k][0], n_p],
                     "n_blocked": [int(res[k][1]["n_blocked"]), int(o["n_blocked"])],
                     "oracle_s": time.perf_counter() - t0})
    out["per_framework"] = rows
    out["max_rel_err"] = max(r["kh_rel_err"] for r in rows) if rows else None
    return out


def cpu_config1_grid():
    """The reference's ComputeGridSheet on the whole config-1 32^3 grid, all
    host cores (seconds)."""
    import oracle
    from emptyroom_b200 import synth
    f = synth.config1(0)
    P = f.particles()
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    if oracle.ref_available():
        oracle.ref_grid(P, f.t_matrix, f.rep, f.rc2, (32, 32, 32), n_threads=cores)
    else:
        oracle.grid(P, f.t_matrix, f.rep, f.rc2, (32, 32, 32), n_threads=cores)
    return time.perf_counter() - t0


def run_config1(ctx):
    """Config 1 as specified: the cubic 25.8 A cell (424 atoms, CH4), its 32^3
    FP64 energy grid and 1e5 Widom insertions at 298 K, each through the C
    ABI with host output (upload included), wall-clocked, best of 5."""
    from emptyroom_b200 import synth
    f = synth.config1(0)
    P = f.particles()
    res = {"workload": "config-1 cell: 32^3 FP64 grid to host + 1e5 Widom insertions, 298 K"}
    tg, th = [], []
    for k in range(6):
        t0 = time.perf_counter()
        fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
        ctx.grid(fw, (32, 32, 32), f64=True)
        t1 = time.perf_counter()
        r = ctx.henry(fw, 298.0, 100_000, seed=k)
        t2 = time.perf_counter()
        fw.release()
        if k:
            tg.append(t1 - t0)
            th.append(t2 - t1)
    res["grid_ms"] = min(tg) * 1e3
    res["henry_ms"] = min(th) * 1e3
    res["kh_mol_m3_pa"] = r["kh_mol_m3_pa"]
    return res


def run_extras(ctx):
    """The remaining rows of the path, one config-4 cell (0.2 A, 129^3):
    GPU pocket blocking (device grid -> device mask), the GCMC grid lookup
    (1e7 guest positions, device in and out), and the parallel .txt grid
    writer (host, byte-identical to the reference's format)."""
    import tempfile

    import torch

    from emptyroom_b200 import files, synth
    f = synth.config4(1, seed=4000)[0]
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    dims = f.dims
    g = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, g.data_ptr())
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    s = torch.cuda.ExternalStream(ctx.stream_ptr)

    def tm(fn, n=5):
        fn()
        ctx.synchronize()
        ts = []
        for _ in range(n):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e-3)
        return min(ts)

    n_p = [0]

    def pockets():
        n_p[0] = ctx.block_pockets_device(g.data_ptr(), dims, 298.0, m.data_ptr())

    t_pk = tm(pockets)
    n_q = 10_000_000
    pts = torch.rand((n_q, 3), dtype=torch.float64, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(0))
    out = torch.empty(n_q, dtype=torch.float64, device="cuda")
    t_lk = tm(lambda: ctx.grid_interp_device(g.data_ptr(), dims, pts.data_ptr(), n_q,
                                             out.data_ptr()))
    host = g.cpu().numpy()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "grid.txt")
        t0 = time.perf_counter()
        files.write_grid_txt(path, host)
        t_io = time.perf_counter() - t0
        size = os.path.getsize(path)
    fw.release()
    return {"workload": f"config-4 cell, 0.2 A grid {list(dims)}",
            "pockets": {"ms": t_pk * 1e3, "n_pockets": n_p[0],
                        "points_per_s": float(np.prod(dims)) / t_pk},
            "gcmc_lookup": {"lookups_per_s": n_q / t_lk, "ms_per_1e7": t_lk * 1e3},
            "grid_txt_write": {"s": t_io, "bytes": size, "mb_per_s": size / t_io / 1e6}}


def cpu_pockets_ref():
    """The reference's FindAndBlockPockets (oracle/_ref) on the same config-4
    grid, computed there by the oracle in FP64 (seconds for the blocking)."""
    import oracle
    from emptyroom_b200 import synth
    f = synth.config4(1, seed=4000)[0]
    E = oracle.grid(f.particles(), f.t_matrix, f.rep, f.rc2, f.dims,
                    n_threads=os.cpu_count() or 1)
    t0 = time.perf_counter()
    if oracle.ref_available():
        oracle.ref_block_pockets(E, 298.0)
    else:
        oracle.block_pockets(E, 298.0)
    return time.perf_counter() - t0


def run_serving(ctx, args):
    """Serving (config 5): a Poisson stream of grid and Henry jobs replayed
    against the request server with 8 slots and against the plain
    one-job-at-a-time loop (1 slot); latency = finish - submit per job. Grid
    jobs leave their grids resident in the server's device cache."""
    from emptyroom_b200 import serve, synth
    fws, jobs = synth.config5_stream(rate=args.serve_rate, seconds=args.serve_seconds)
    descs = [serve.framework_desc(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws]

    def schedule():
        out = []
        for j in jobs:
            d = descs[j["fw"]]
            if j["kind"] == "grid":
                out.append((j["t"], lambda srv, j=j, d=d: srv.submit_grid(j["fw"], d, j["dims"])))
            else:
                out.append((j["t"], lambda srv, j=j, d=d: srv.submit_henry(
                    j["fw"], d, 298.0, j["n_ins"], j["seed"])))
        return out

    res = {"workload": f"Poisson {len(jobs)} jobs over {args.serve_seconds:.0f} s "
                       f"({len(jobs) / args.serve_seconds:.0f} jobs/s; 70% grid, 30% Henry "
                       f"1e6-1e7 insertions; {len(fws)} frameworks; config 5)",
           "hbm_budget_gib": args.serve_budget_gib}
    for name, slots in (("served", 8), ("plain", 1)):
        with serve.Server(ctx, int(args.serve_budget_gib * (1 << 30)), slots) as srv:
            # atom arrays resident first (one small Henry job per framework)
            for k, d in enumerate(descs):
                srv.wait(srv.submit_henry(k, d, 298.0, 1000, 0))
            t0 = time.perf_counter()
            sts = serve.run_stream(srv, schedule())
            wall = time.perf_counter() - t0
        lat = np.array([st["latency_s"] for st in sts], dtype=np.float64) * 1e3
        wait = np.array([st["start_s"] - st["submit_s"] for st in sts]) * 1e3
        serv = np.array([st["finish_s"] - st["start_s"] for st in sts]) * 1e3
        kinds = np.array([j["kind"] for j in jobs])
        res[name] = {"slots": slots, "p50_ms": float(np.percentile(lat, 50)),
                     "p99_ms": float(np.percentile(lat, 99)),
                     "queue_wait_p50_ms": float(np.percentile(wait, 50)),
                     "queue_wait_p99_ms": float(np.percentile(wait, 99)),
                     "service_p50_ms": float(np.percentile(serv, 50)),
                     "service_p99_ms": float(np.percentile(serv, 99)),
                     "grid_p50_ms": float(np.percentile(lat[kinds == "grid"], 50)),
                     "henry_p50_ms": float(np.percentile(lat[kinds == "henry"], 50)),
                     "jobs_per_s": len(sts) / wall,
                     "failed": int(sum(1 for st in sts if st["status"] != 0))}
    return res


def load_traffic(points_step):
    """DRAM bytes per launch of the persistent kernel from the committed ncu
    capture of a smaller batch (profiles/grid_persistent_traffic.json), scaled
    to this launch by grid points (the traffic is the grid store)."""
    p = os.path.join(ROOT, "profiles", "grid_persistent_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d["dram_bytes_per_point"] * points_step


def run_reference(args, ws, rank):
    """The reference's own CPU implementation on the host cores: its
    ComputeGridSheet (oracle/_ref, compiled from its sources) on a bounded
    sample of the batch's grids each step, and its LJ routine at Widom
    insertion points. The frameworks come from oracle/workloads.py (this
    library is not loaded)."""
    import oracle
    from oracle import workloads
    if rank != 0:
        return None
    fws = workloads.config2(256)
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(11)
    step_target = 3.0
    values, step_s = [], []
    samples = []
    for step in range(args.warmup + args.steps):
        pairs, secs, sample = ref_grid_sample(fws, step_target, rng, cores)
        if step == 0:
            samples = sample
        if step >= args.warmup:
            values.append(pairs / secs)
            step_s.append(secs)
    n_ins, wpairs, wsecs = ref_widom_sample(workloads.config4(1)[0], 6.0, cores)
    v = float(np.mean(values))
    kind = "reference" if oracle.ref_available() else "port"
    return {"metric": METRIC, "value": v, "unit": "pair-terms/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(step_s)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded frameworks)", "impl": "reference",
            "config": {"workload": WORKLOAD,
                       "sample": "each step: random grid points of randomly chosen "
                                 f"frameworks of the batch, ~{step_target:.0f} s of the "
                                 "reference's ComputeGridSheet on all host cores"},
            "cpu_baseline": {"value": v, "unit": "pair-terms/s", "cores": cores, "kind": kind,
                             "sample": f"256-point chunks of frameworks {samples[:6]}..., "
                                       f"~{step_target:.0f} s per step"},
            "widom": {"insertions_per_s": n_ins / wsecs, "pair_terms_per_s": wpairs / wsecs,
                      "sample": f"first {n_ins} Philox insertions of a config-4 cell (Xe), "
                                "the reference's LJ routine at each point"},
            "e2e": {"value": v, "unit": "pair-terms/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def case_precision(ctx, args):
    """Precision sweep on the config-3 cell (30.1, 32.4, 28.7 A; 85/95/110 deg;
    CH4; cutoff 12.5 A) on a dims^3 grid, 4096 atoms as specified or
    --atoms (646 gives the config-1 number density): the ER_PREC_FP32,
    ER_PREC_COMP and default (NEAR64) grids against the ER_PREC_FP64 grid,
    itself pinned to the oracle on sampled points."""
    import emptyroom_b200 as er
    import oracle
    from emptyroom_b200 import synth
    f = synth.config3() if args.atoms == 4096 else synth.make_framework(
        3, (30.1, 32.4, 28.7), (85.0, 95.0, 110.0), args.atoms, n_types=4, probe="CH4",
        rc=12.5, d_min=1.2, name=f"config3_{args.atoms}")
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = (args.dims,) * 3
    e64 = ctx.grid(fw, dims, precision=er.ER_PREC_FP64, f64=True)
    rng = np.random.default_rng(7)
    idx = rng.integers(0, args.dims, size=(4000, 3))
    pts = idx / (args.dims - 1.0)
    ref, S, _ = oracle.points_cells(P, f.t_matrix, f.rep, f.rc2, pts, 1e-12)
    got = e64[idx[:, 0], idx[:, 1], idx[:, 2]]
    ok = ref < er.ER_ENERGY_CAP
    res = {"workload": f"config-3 cell, {args.atoms} atoms, {args.dims}^3 grid, CH4, rc 12.5 A",
           "fp64_grid_vs_oracle_max_over_sum_abs": float(
               np.max(np.abs(got[ok] - ref[ok]) / np.maximum(S[ok], 1e-300))),
           "modes": {}}

    def stats(e):
        e = e.astype(np.float64)
        out = {"cap_agrees": bool(np.array_equal(e >= er.ER_ENERGY_CAP, e64 >= er.ER_ENERGY_CAP))}
        for name, msk in (("neg", e64 < 0), ("below_-1K", e64 < -1.0),
                          ("below_-10K", e64 < DEEP), ("pos", (e64 >= 0) & (e64 < 1e10))):
            d = np.abs(e[msk] - e64[msk])
            r = d / np.maximum(np.abs(e64[msk]), 1e-30)
            out[name] = {"n": int(msk.sum()),
                         "abs_max": float(d.max()) if d.size else 0.0,
                         "abs_p99": float(np.percentile(d, 99)) if d.size else 0.0,
                         "rel_max": float(r.max()) if r.size else 0.0,
                         "rel_p99": float(np.percentile(r, 99)) if r.size else 0.0,
                         "frac_rel_le_1e-5": float(np.mean(r <= 1e-5)) if r.size else 1.0}
        return out

    for name, flags in (("fp32", er.ER_PREC_FP32), ("comp", er.ER_PREC_COMP),
                        ("near64_default", er.ER_PREC_NEAR64)):
        res["modes"][name] = stats(ctx.grid(fw, dims, precision=flags))
    fw.release()
    print(json.dumps(res, indent=1))


def case_refgpu(ctx, args):
    """The reference's own GPU writegrid (oracle/_ref/writegrid, its sources
    compiled for sm_100a) beside this library on the same B200 and case: the
    config-1 cell at 0.2 A (129^3 points). Writes the project tree the
    reference reads into --tree and prints this library's grid time (CUDA
    events, er_grid into device memory) and the exact pair count; the
    reference's kernel times come from an ncu launch list of its writegrid
    run in that tree."""
    import torch

    from emptyroom_b200 import synth
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fixture_tree import write_tree
    f = synth.config1(0)
    name, ads = write_tree(args.tree, f, resolution=0.2)
    dims = synth.grid_dims_for(f.abc, 0.2)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    out = torch.empty(dims, dtype=torch.float32, device="cuda")
    s = torch.cuda.ExternalStream(ctx.stream_ptr)
    ts = []
    for k in range(6):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.grid_device(fw, dims, out.data_ptr())
        e1.record(s)
        e1.synchronize()
        if k >= 2:
            ts.append(e0.elapsed_time(e1) * 1e-3)
    ctx.count_pairs_device(fw, dims, out.data_ptr())
    ctx.synchronize()
    pairs = float(out.double().sum().item())
    t = min(ts)
    print(json.dumps({"framework": name, "adsorbate": ads, "dims": list(dims), "pairs": pairs,
                      "ours_s": t, "ours_pair_terms_per_s": pairs / t}))


def run_case(args):
    """Single-kernel and analysis cases: `config3` runs the 4096-atom triclinic
    cell on a dims^3 grid (one er_grid launch per step); `widom` runs er_henry
    with --insertions points on a config-1 cell; `widom_batch` er_henry_batch
    over --widom-frameworks config-4 cells (pocket grid, device mask and
    --insertions points each); `precision` the precision sweep; `refgpu` this
    library beside the reference's own GPU writegrid."""
    import torch

    import emptyroom_b200 as er
    from emptyroom_b200 import synth
    ctx = er.Context(0)
    if args.case == "precision":
        case_precision(ctx, args)
    elif args.case == "refgpu":
        case_refgpu(ctx, args)
    elif args.case == "config3":
        f = synth.config3()
        fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
        dims = (args.dims,) * 3
        out = torch.empty(dims, dtype=torch.float32, device="cuda")
        s = torch.cuda.ExternalStream(ctx.stream_ptr)
        flags = (er.ER_TILE_P8 if args.tile == 8 else 0) | \
            (er.ER_PREC_COMP if args.precision == "comp" else 0)
        times = []
        for k in range(args.warmup + args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            ctx.grid_device(fw, dims, out.data_ptr(), precision=flags)
            e1.record(s)
            e1.synchronize()
            if k >= args.warmup:
                times.append(e0.elapsed_time(e1) * 1e-3)
        cnt = torch.empty(dims, dtype=torch.float32, device="cuda")
        ctx.count_pairs_device(fw, dims, cnt.data_ptr())
        ctx.synchronize()
        pairs = float(cnt.double().sum().item())
        t = sum(times) / len(times)
        print(json.dumps({"case": "config3", "dims": dims, "tile_p": args.tile,
                          "precision": args.precision, "ms": t * 1e3, "pairs": pairs,
                          "pair_terms_per_s": pairs / t,
                          "pairs_per_point": pairs / float(np.prod(dims))}))
    elif args.case == "widom_batch":
        fws = synth.config4(args.widom_frameworks)
        ups = ctx.upload_many([(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws])
        dims = fws[0].dims
        times = []
        for k in range(args.warmup + args.steps):
            seeds = [k * len(ups) + j for j in range(len(ups))]
            ctx.synchronize()
            t0 = time.perf_counter()
            res, _ = ctx.henry_batch(ups, 298.0, args.insertions, seeds, block_dims=dims)
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        t = sum(times) / len(times)
        n_ins = args.insertions * len(ups)
        print(json.dumps({"case": "widom_batch", "frameworks": len(ups), "dims": list(dims),
                          "insertions": n_ins, "ms": t * 1e3, "insertions_per_s": n_ins / t}))
    else:
        f = synth.make_framework(0, (25.8, 25.8, 25.8), (90, 90, 90), 424, probe="Xe")
        fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
        times = []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            r = ctx.henry(fw, 298.0, args.insertions, seed=k)
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        t = sum(times) / len(times)
        print(json.dumps({"case": "widom", "insertions": args.insertions, "ms": t * 1e3,
                          "insertions_per_s": args.insertions / t, "kh": r["kh_mol_m3_pa"]}))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-errors", action="store_true",
                    help="skip the oracle comparison of the grids and K_H")
    ap.add_argument("--case", default="batch",
                    choices=["batch", "config3", "widom", "widom_batch", "precision", "refgpu"])
    ap.add_argument("--dims", type=int, default=256)
    ap.add_argument("--atoms", type=int, default=4096)
    ap.add_argument("--tree", default="/tmp/er_tree")
    ap.add_argument("--insertions", type=int, default=10_000_000)
    ap.add_argument("--tile", type=int, default=4, choices=[4, 8])
    ap.add_argument("--precision", default="near64", choices=["near64", "comp"])
    ap.add_argument("--frameworks", type=int, default=256,
                    help="frameworks of the batch (256 is the workload; fewer for profiling)")
    ap.add_argument("--no-widom", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--widom-frameworks", type=int, default=64)
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="length of the Poisson stream (config 5: 60 s)")
    ap.add_argument("--serve-budget-gib", type=float, default=48.0)
    ap.add_argument("--serve-rate", type=float, default=200.0,
                    help="mean arrivals per second of the Poisson stream (config 5: 200)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.case != "batch":
        run_case(args)
        return
    ws, rank, local, pg = dist_setup()
    if args.impl == "reference":
        line = run_reference(args, ws, rank)
    else:
        line = run_ours(args, ws, rank, local, pg)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
