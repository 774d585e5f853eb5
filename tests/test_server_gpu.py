"""The request server (er_server_*): results identical alone and in the mix,
HBM-budget admission with eviction, the device-resident grid cache, the
one-slot plain loop, bounded waits."""
import numpy as np
import pytest

from emptyroom_b200 import serve, synth

pytestmark = pytest.mark.gpu


def _frameworks(n=4, seed=300):
    out = []
    for k in range(n):
        f = synth.make_framework(seed + k, (14.0 + 2 * k, 15.0, 13.5 + k), (85, 95, 100),
                                 60 + 40 * k, probe=["CH4", "Xe", "Kr"][k % 3], rc=12.5)
        desc = serve.framework_desc(f.particles(), f.t_matrix, f.rep, f.rc2)
        out.append((f, desc))
    return out


def _pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float32, pin_memory=True)


def test_results_same_alone_and_in_mix(ctx):
    fws = _frameworks()
    dims = [(20, 22, 18), (31, 17, 25), (16, 16, 40), (27, 27, 27)]
    bufs = [_pinned(d) for d in dims]
    with serve.Server(ctx, 8 << 30, slots=4) as srv:
        tickets = []
        for k, ((f, desc), d, b) in enumerate(zip(fws, dims, bufs)):
            tickets.append(("g", k, srv.submit_grid(k, desc, d, b.data_ptr())))
            tickets.append(("h", k, srv.submit_henry(k, desc, 298.0, 30000 + 7 * k, k + 1)))
        res = {(kind, k): srv.wait(t) for kind, k, t in tickets}
    for (kind, k), st in res.items():
        assert st["done"] and st["status"] == 0, st
    # now each job alone, through the ordinary entry points
    for k, ((f, desc), d, b) in enumerate(zip(fws, dims, bufs)):
        fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
        assert np.array_equal(b.numpy(), ctx.grid(fw, d))
        h = ctx.henry(fw, 298.0, 30000 + 7 * k, seed=k + 1)
        assert res[("h", k)]["henry"]["sum_w"] == h["sum_w"]
        assert res[("h", k)]["henry"]["kh_mol_m3_pa"] == h["kh_mol_m3_pa"]
        fw.release()


def test_plain_loop_matches_batched(ctx):
    fws = _frameworks(3, seed=320)
    dims = (24, 20, 22)
    outs = {}
    for slots in (1, 3):
        bufs = [_pinned(dims) for _ in fws]
        with serve.Server(ctx, 8 << 30, slots=slots) as srv:
            ts = [srv.submit_grid(k, desc, dims, b.data_ptr()) for k, ((f, desc), b) in
                  enumerate(zip(fws, bufs))]
            for t in ts:
                assert srv.wait(t)["status"] == 0
        outs[slots] = [b.numpy().copy() for b in bufs]
    for a, b in zip(outs[1], outs[3]):
        assert np.array_equal(a, b)


def test_grid_cache_and_eviction(ctx):
    fws = _frameworks(2, seed=340)
    dims = (40, 40, 40)  # 256 KB per grid
    grid_bytes = 40 ** 3 * 4
    with serve.Server(ctx, 8 << 30, slots=2) as srv:
        reserved = srv.device_bytes  # the slots' Widom scratch, reserved at creation
        b1 = _pinned(dims)
        t1 = srv.submit_grid(7, fws[0][1], dims, b1.data_ptr())
        s1 = srv.wait(t1)
        b2 = _pinned(dims)
        t2 = srv.submit_grid(7, fws[0][1], dims, b2.data_ptr())
        s2 = srv.wait(t2)
        assert s1["grid_cache_hit"] == 0 and s2["grid_cache_hit"] == 1
        assert np.array_equal(b1.numpy(), b2.numpy())
        assert srv.grid_ptr(t1) == srv.grid_ptr(t2)
        assert srv.device_bytes >= grid_bytes
        # what both frameworks cost when resident (plus a 2^3 grid)
        t3 = srv.submit_grid(8, fws[1][1], (2, 2, 2))
        srv.wait(t3)
        fw_bytes = srv.device_bytes - grid_bytes - reserved
    # a budget that holds both frameworks but only about two grids at a time
    small = fw_bytes + int(2.5 * grid_bytes)
    with serve.Server(ctx, small, slots=2) as srv:
        ts, keep = [], []
        for k in range(6):
            dk = (40, 40, 40 - k)
            keep.append(_pinned(dk))  # host buffers must outlive their jobs
            ts.append(srv.submit_grid(10 + k % 2, fws[k % 2][1], dk, keep[-1].data_ptr()))
        for t in ts:
            assert srv.wait(t)["status"] == 0
        assert srv.device_bytes <= small
        # the oldest grids were evicted, the newest is resident
        with pytest.raises(serve.ServerError):
            srv.grid_ptr(ts[0])
        srv.grid_ptr(ts[-1])
    # with the budget full, later grids take over evicted grids' buffers
    # (slightly larger ones): every result is still the single call's
    ups = [ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2) for f, _ in fws]
    for k in range(6):
        dk = (40, 40, 40 - k)
        assert np.array_equal(keep[k].numpy(), ctx.grid(ups[k % 2], dk))
    for u in ups:
        u.release()


def test_job_larger_than_budget_fails_cleanly(ctx):
    fws = _frameworks(1, seed=360)
    with serve.Server(ctx, 1 << 20, slots=1) as srv:
        t = srv.submit_grid(1, fws[0][1], (200, 200, 200))
        st = srv.wait(t)
        assert st["done"] and st["status"] == 3  # ER_ERR_NOMEM
        t2 = srv.submit_grid(1, fws[0][1], (10, 10, 10))
        assert srv.wait(t2)["status"] == 0


def test_wait_timeout_is_bounded(ctx):
    fws = _frameworks(1, seed=370)
    with serve.Server(ctx, 8 << 30, slots=1) as srv:
        big = srv.submit_henry(1, fws[0][1], 298.0, 3_000_000, 5)
        small = srv.submit_grid(1, fws[0][1], (12, 12, 12))
        with pytest.raises(TimeoutError):
            srv.wait(small, timeout=0.0)
        assert srv.wait(big)["status"] == 0
        assert srv.wait(small)["status"] == 0


def test_poisson_stream_latencies(ctx):
    fws = _frameworks(3, seed=380)
    rng = np.random.default_rng(0)
    arrivals = np.cumsum(rng.exponential(1 / 200.0, size=60))
    schedule = []
    for k, a in enumerate(arrivals):
        f, desc = fws[k % 3]
        if rng.random() < 0.7:
            d = tuple(int(x) for x in rng.integers(20, 48, size=3))
            schedule.append((a, lambda s, d=d, k=k, desc=desc: s.submit_grid(k % 3, desc, d)))
        else:
            n = int(rng.integers(20000, 200000))
            schedule.append((a, lambda s, n=n, k=k, desc=desc: s.submit_henry(k % 3, desc, 298.0,
                                                                             n, k)))
    with serve.Server(ctx, 8 << 30, slots=8) as srv:
        sts = serve.run_stream(srv, schedule)
    lat = np.array([s["latency_s"] for s in sts])
    assert all(s["status"] == 0 for s in sts)
    assert np.all(lat >= 0) and np.percentile(lat, 50) < 1.0
