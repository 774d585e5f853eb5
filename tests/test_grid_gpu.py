"""Parity of the CUDA grid path (er_grid and friends, through the C ABI) with
the reference's FP64 results: the golden fixtures, the oracle at full grids
of small cells, and the oracle at sampled points of large grids."""
import numpy as np
import pytest

import emptyroom_b200 as er
import oracle
from conftest import golden, grid_errors, rotated_cell
from emptyroom_b200 import synth

pytestmark = pytest.mark.gpu


def _check(stats):
    assert stats["neg_ok"], stats
    assert stats["pos_ok"], stats
    assert stats["cap_ok"], stats


@pytest.mark.parametrize("name", ["grid_cubic", "grid_triclinic", "grid_rep2"])
def test_grid_matches_golden(ctx, name):
    g = golden(name)
    fw = ctx.upload(g["particles"], g["t_matrix"], g["rep"], float(g["rc2"]))
    e = ctx.grid(fw, g["dims"])
    S = oracle.grid_abs(g["particles"], g["t_matrix"], g["rep"], float(g["rc2"]), g["dims"])
    _check(grid_errors(e, g["grid"], S))
    fw.release()


def test_grid_config1_full(ctx):
    fw_s = synth.config1(0)
    P = fw_s.particles()
    fw = ctx.upload(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    e = ctx.grid(fw, (32, 32, 32))
    ref = oracle.grid(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, (32, 32, 32))
    S = oracle.grid_abs(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, (32, 32, 32))
    st = grid_errors(e, ref, S)
    _check(st)
    assert st["n_neg"] > 0


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_grid_triclinic_odd_sizes(ctx, seed):
    rng = np.random.default_rng(seed)
    abc = tuple(rng.uniform(9, 30, size=3))
    ang = tuple(rng.uniform(65, 115, size=3))
    n = int(rng.integers(20, 300))
    fw_s = synth.make_framework(seed, abc, ang, n, probe=["CH4", "Xe", "Kr"][seed % 3])
    dims = tuple(int(x) for x in rng.integers(2, 23, size=3))
    P = fw_s.particles()
    fw = ctx.upload(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    e = ctx.grid(fw, dims)
    ref = oracle.grid(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, dims)
    S = oracle.grid_abs(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, dims)
    _check(grid_errors(e, ref, S))


def test_grid_large_sampled_points(ctx):
    """config-3 cell (4096 atoms) on a 96^3 grid: 3000 sampled points vs the oracle."""
    fw_s = synth.config3()
    P = fw_s.particles()
    fw = ctx.upload(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    dims = (96, 96, 96)
    e = ctx.grid(fw, dims)
    rng = np.random.default_rng(0)
    idx = rng.integers(0, np.array(dims), size=(3000, 3))
    pts = idx / (np.array(dims) - 1.0)
    ref = oracle.points(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, pts, 1e-12)
    S = oracle.points_abs(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, pts, 1e-12)
    _check(grid_errors(e[idx[:, 0], idx[:, 1], idx[:, 2]], ref, S))


def test_sheet_and_f64_and_device_outputs_agree(ctx):
    import torch
    fw_s = synth.config1(3)
    fw = ctx.upload(fw_s.particles(), fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    dims = (17, 18, 19)
    e32 = ctx.grid(fw, dims)
    e64 = ctx.grid(fw, dims, f64=True)
    assert e64.dtype == np.float64 and np.array_equal(e64, e32.astype(np.float64))
    for i in (0, 7, 16):
        assert np.array_equal(ctx.grid_sheet(fw, dims, i), e32[i].astype(np.float64))
    d = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, d.data_ptr())
    ctx.synchronize()
    assert np.array_equal(d.cpu().numpy(), e32)
    d64 = torch.empty(dims, dtype=torch.float64, device="cuda")
    ctx.grid_device(fw, dims, d64.data_ptr(), f64=True)
    ctx.synchronize()
    assert np.array_equal(d64.cpu().numpy(), e64)


def test_grid_is_deterministic(ctx):
    fw_s = synth.config1(4)
    fw = ctx.upload(fw_s.particles(), fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    a = ctx.grid(fw, (33, 31, 29))
    b = ctx.grid(fw, (33, 31, 29))
    assert np.array_equal(a, b)


def test_fp32_mode_close(ctx):
    fw_s = synth.config1(5)
    P = fw_s.particles()
    fw = ctx.upload(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    dims = (20, 20, 20)
    e = ctx.grid(fw, dims, precision=er.ER_PREC_FP32)
    ref = oracle.grid(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, dims)
    S = oracle.grid_abs(P, fw_s.t_matrix, fw_s.rep, fw_s.rc2, dims)
    neg = ref < 0
    assert np.all(np.abs(e[neg] - ref[neg]) <= 1e-5 * np.abs(ref[neg]) + 1e-5 * S[neg])


def test_invalid_arguments(ctx):
    fw_s = synth.config1(6)
    fw = ctx.upload(fw_s.particles(), fw_s.t_matrix, fw_s.rep, fw_s.rc2)
    with pytest.raises(er.ErError):
        ctx.grid(fw, (1, 8, 8))
    with pytest.raises(er.ErError):
        ctx.upload(fw_s.particles(), fw_s.t_matrix, fw_s.rep, -1.0)
    bad = er.Framework(ctx, 987654, 0)
    with pytest.raises(er.ErError):
        ctx.grid(bad, (4, 4, 4))


def test_empty_framework_gives_zero(ctx):
    t, _, _ = er.cell_matrices(10, 10, 10, 90, 90, 90)
    fw = ctx.upload(np.zeros((0, 5)), t, (1, 1, 1), 100.0)
    e = ctx.grid(fw, (5, 5, 5))
    assert np.all(e == 0)


def test_point_on_atom_is_capped(ctx):
    """A grid point exactly on an atom: the reference gives an astronomically
    large finite value; the CUDA path writes the overflow cap."""
    t, _, _ = er.cell_matrices(10, 10, 10, 90, 90, 90)
    P = er.particles([[0.5, 0.5, 0.5], [0.1, 0.2, 0.3]], [50.0, 60.0], [9.0, 10.0])
    fw = ctx.upload(P, t, (1, 1, 1), 25.0)
    dims = (3, 3, 3)  # the centre point (1,1,1) sits on atom 0
    e = ctx.grid(fw, dims)
    ref = oracle.grid(P, t, (1, 1, 1), 25.0, dims)
    assert ref[1, 1, 1] > 1e30 and e[1, 1, 1] == np.float32(1e30)
    _check(grid_errors(e, ref, oracle.grid_abs(P, t, (1, 1, 1), 25.0, dims)))


def _batch_frameworks(ctx, n=12, seed=50):
    fws = synth.config2(n_frameworks=n, seed=seed, spacing_range=(0.9, 1.6))
    ups = [ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws]
    return fws, ups


def test_batch_modes_identical_and_match_single(ctx):
    import torch
    fws, ups = _batch_frameworks(ctx)
    outs_p = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    outs_q = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs_p)],
                   er.ER_BATCH_PERSISTENT)
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs_q)],
                   er.ER_BATCH_PLAIN)
    for u, f, a, b in zip(ups, fws, outs_p, outs_q):
        single = ctx.grid(u, f.dims)
        assert np.array_equal(a.cpu().numpy(), single)
        assert np.array_equal(b.cpu().numpy(), single)


def test_batch_alone_equals_in_mix(ctx):
    import torch
    fws, ups = _batch_frameworks(ctx, n=10, seed=77)
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)])
    k = 4
    alone = torch.empty(fws[k].dims, dtype=torch.float32, device="cuda")
    ctx.grid_batch([(ups[k], fws[k].dims, alone.data_ptr())])
    assert torch.equal(alone, outs[k])


def test_batch_plan_graph_replay(ctx):
    import torch
    fws, ups = _batch_frameworks(ctx, n=6, seed=91)
    outs = [torch.zeros(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    plan = ctx.batch_plan([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)])
    assert plan.launches == 1
    plan.run()
    ctx.synchronize()
    first = [o.clone() for o in outs]
    for o in outs:
        o.zero_()
    torch.cuda.synchronize()  # the zeroing runs on torch's stream, the plan on the library's
    plan.run()
    ctx.synchronize()
    for a, b in zip(first, outs):
        assert torch.equal(a, b)
    plain = ctx.batch_plan([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)],
                           er.ER_BATCH_PLAIN)
    assert plain.launches == len(fws)
    plan.close()
    plain.close()


def test_batch_matches_oracle_sampled(ctx):
    import torch
    fws, ups = _batch_frameworks(ctx, n=5, seed=123)
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)])
    rng = np.random.default_rng(1)
    for f, o in zip(fws, outs):
        dims = np.array(f.dims)
        idx = rng.integers(0, dims, size=(200, 3))
        pts = idx / (dims - 1.0)
        ref = oracle.points(f.particles(), f.t_matrix, f.rep, f.rc2, pts, 1e-12)
        S = oracle.points_abs(f.particles(), f.t_matrix, f.rep, f.rc2, pts, 1e-12)
        got = o.cpu().numpy()[idx[:, 0], idx[:, 1], idx[:, 2]]
        _check(grid_errors(got, ref, S))


@pytest.mark.parametrize("name", ["grid_cubic", "grid_triclinic", "grid_rep2"])
def test_accessibility_matches_golden(ctx, name):
    g = golden(name)
    fw = ctx.upload(g["particles"], g["t_matrix"], g["rep"], float(g["rc2"]))
    a = ctx.accessibility(fw, g["dims"])
    assert np.array_equal(a, g["accessibility"])


def test_accessibility_matches_oracle_config1(ctx):
    f = synth.config1(9)
    P = f.particles()
    P[::7, 3] = 0.0  # epsilon = 0 atoms still occupy space in the hard-sphere test
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    a = ctx.accessibility(fw, (40, 33, 29))
    assert np.array_equal(a, oracle.accessibility(P, f.t_matrix, (40, 33, 29)))


def test_autotuned_plan_matches_er_grid_with_its_variant(ctx):
    import torch
    fws, ups = _batch_frameworks(ctx, n=8, seed=140)
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    plan = ctx.batch_plan([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)],
                          er.ER_BATCH_PERSISTENT | er.ER_BATCH_AUTOTUNE)
    plan.run()
    ctx.synchronize()
    for k, (u, f, o) in enumerate(zip(ups, fws, outs)):
        p = plan.tile(k)
        assert p in (4, 8)
        flags = er.ER_TILE_P8 if p == 8 else 0
        assert np.array_equal(o.cpu().numpy(), ctx.grid(u, f.dims, precision=flags))
    plan.close()


@pytest.mark.parametrize("flags", [er.ER_TILE_P8, er.ER_PREC_COMP,
                                   er.ER_PREC_COMP | er.ER_TILE_P8])
def test_variants_match_oracle(ctx, flags):
    f = synth.make_framework(150, (17.0, 19.0, 18.0), (80, 100, 95), 120, probe="Xe")
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = (27, 19, 33)
    e = ctx.grid(fw, dims, precision=flags)
    ref = oracle.grid(P, f.t_matrix, f.rep, f.rc2, dims)
    S = oracle.grid_abs(P, f.t_matrix, f.rep, f.rc2, dims)
    _check(grid_errors(e, ref, S, loose=bool(flags & er.ER_PREC_COMP)))


def test_near64_is_more_accurate_than_comp(ctx):
    f = synth.config1(7)
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = (30, 30, 30)
    ref = oracle.grid(P, f.t_matrix, f.rep, f.rc2, dims)
    neg = ref < 0
    e32 = ctx.grid(fw, dims, precision=er.ER_PREC_COMP).astype(np.float64)
    e64 = ctx.grid(fw, dims).astype(np.float64)
    err32 = np.abs(e32 - ref)[neg].max()
    err64 = np.abs(e64 - ref)[neg].max()
    # NEAR64 errors are left by the FP32 far pairs and the FP32 output rounding
    assert err64 < err32
    assert np.all(np.abs(e64 - ref)[neg] <= 2e-6 * np.abs(ref[neg]) + 2e-4)


_rotated = rotated_cell


@pytest.mark.parametrize("flags", [0, er.ER_TILE_P8])
def test_rotated_cell_matches_oracle(ctx, flags):
    f = synth.make_framework(160, (16.0, 19.0, 17.5), (75, 105, 98), 140, probe="Kr")
    P = f.particles()
    t = _rotated(f.t_matrix, 3)
    assert abs(t[1, 0]) > 1e-3 and abs(t[2, 0]) > 1e-3
    fw = ctx.upload(P, t, f.rep, f.rc2)
    dims = (21, 18, 26)
    e = ctx.grid(fw, dims, precision=flags)
    ref = oracle.grid(P, t, f.rep, f.rc2, dims)
    S = oracle.grid_abs(P, t, f.rep, f.rc2, dims)
    _check(grid_errors(e, ref, S))
    # the summed pair set is the reference's, exactly
    cnt = ctx.count_pairs(fw, dims)
    want = oracle.points_pairs(P, t, f.rep, f.rc2, oracle.lattice_points(dims))
    assert np.array_equal(cnt.astype(np.float64).ravel(), want)


@pytest.mark.parametrize("flags", [0, er.ER_TILE_P8])
def test_pair_counts_exact(ctx, flags):
    f = synth.config1(3)
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = (23, 31, 17)
    cnt = ctx.count_pairs(fw, dims) if flags == 0 else None
    if cnt is None:
        cnt = np.empty(dims, dtype=np.float32)
        import ctypes
        from emptyroom_b200 import _capi
        assert _capi.lib().er_grid(ctx._h, fw.id, *dims, er.ER_COUNT_PAIRS | flags,
                                   cnt.ctypes.data_as(ctypes.c_void_p)) == 0
    want = oracle.points_pairs(P, f.t_matrix, f.rep, f.rc2, oracle.lattice_points(dims))
    assert np.array_equal(cnt.astype(np.float64).ravel(), want)


@pytest.mark.parametrize("flags", [0, er.ER_TILE_P8])
def test_fp64_mode_matches_oracle(ctx, flags):
    f = synth.make_framework(170, (18.0, 17.0, 21.0), (88, 100, 93), 160, probe="CH4")
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = (19, 22, 15)
    e = ctx.grid(fw, dims, precision=er.ER_PREC_FP64 | flags, f64=True)
    ref = oracle.grid(P, f.t_matrix, f.rep, f.rc2, dims)
    S = oracle.grid_abs(P, f.t_matrix, f.rep, f.rc2, dims)
    cap = ref >= er.ER_ENERGY_CAP
    assert np.array_equal(e >= er.ER_ENERGY_CAP, cap)
    ok = ~cap
    # FP64 terms summed in another order (and positions relative to a box
    # centre): errors of a few ulps of the absolute sum
    assert np.all(np.abs(e[ok] - ref[ok]) <= 1e-12 * S[ok] + 1e-9)


def test_fp64_mode_needs_f64_output(ctx):
    f = synth.config1(0)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    with pytest.raises(er.ErError):
        ctx.grid(fw, (4, 4, 4), precision=er.ER_PREC_FP64)


@pytest.mark.parametrize("mode", [er.ER_BATCH_PERSISTENT, er.ER_BATCH_PLAIN,
                                  er.ER_BATCH_PERSISTENT | er.ER_BATCH_AUTOTUNE])
def test_batch_host_out_matches_device(ctx, mode):
    """HOST_OUT copies each grid back while the kernel still runs (persistent
    mode); the host grids equal the device-batch grids bit for bit."""
    import torch
    fws, ups = _batch_frameworks(ctx, n=14, seed=120)
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)],
                   mode & ~er.ER_BATCH_HOST_OUT)
    hosts = [torch.full(f.dims, float("nan"), dtype=torch.float32, pin_memory=True)
             for f in fws]
    for rep in range(2):  # the second call reuses the flag and staging buffers
        for h in hosts:
            h.fill_(float("nan"))
        ctx.grid_batch([(u, f.dims, h.data_ptr()) for u, f, h in zip(ups, fws, hosts)],
                       mode | er.ER_BATCH_HOST_OUT)
        for o, h in zip(outs, hosts):
            assert torch.equal(o.cpu(), h)


def test_upload_many_equals_single_uploads(ctx):
    fws = synth.config2(n_frameworks=9, seed=130, spacing_range=(0.9, 1.6))
    many = ctx.upload_many([(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws])
    assert len({u.id for u in many}) == len(fws)
    for f, u in zip(fws, many):
        single = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
        assert u.device_bytes == single.device_bytes
        assert np.array_equal(ctx.grid(u, f.dims), ctx.grid(single, f.dims))
        single.release()
    for u in many:
        u.release()


def test_upload_many_device_build_edge_cases(ctx):
    """er_framework_upload_many builds the image cell lists on the device;
    er_framework_upload builds them on the host. The two blocks must be the
    same on the cases the builder branches on: no atoms, atoms with eps == 0
    (no images), a small cell with large replication, a rotated (not upper
    triangular) cell matrix, and a call with a single framework."""
    small = synth.make_framework(171, (8.2, 9.0, 8.6), (70, 110, 95), 30, probe="Xe")
    base = synth.make_framework(172, (16.0, 19.0, 17.5), (75, 105, 98), 140, probe="Kr")
    P = base.particles()
    no_eps = P.copy()
    no_eps[::3, 3] = 0.0  # every third atom: eps == 0
    items = [
        (P[:0], base.t_matrix, base.rep, base.rc2),
        (no_eps, base.t_matrix, base.rep, base.rc2),
        (small.particles(), small.t_matrix, small.rep, small.rc2),
        (P, _rotated(base.t_matrix, 5), base.rep, base.rc2),
    ]
    assert max(small.rep) >= 2
    dims = (13, 11, 15)
    for batch in (items, items[3:]):
        many = ctx.upload_many(batch)
        for it, u in zip(batch, many):
            single = ctx.upload(*it)
            assert u.device_bytes == single.device_bytes
            assert np.array_equal(ctx.grid(u, dims), ctx.grid(single, dims))
            assert np.array_equal(ctx.count_pairs(u, dims), ctx.count_pairs(single, dims))
            assert np.array_equal(ctx.grid(u, dims, precision=er.ER_PREC_COMP),
                                  ctx.grid(single, dims, precision=er.ER_PREC_COMP))
            single.release()
        for u in many:
            u.release()
    assert not ctx.grid(ctx.upload_many(items[:1])[0], dims).any()


def test_upload_many_reports_the_bad_framework(ctx):
    fws = synth.config2(n_frameworks=3, seed=131, spacing_range=(0.9, 1.6))
    items = [(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws]
    bad = items[1][0].copy()
    bad[0, 3] = -1.0  # negative epsilon
    items[1] = (bad,) + items[1][1:]
    with pytest.raises(er.ErError, match="framework 1"):
        ctx.upload_many(items)


@pytest.mark.parametrize("mode", [er.ER_BATCH_PERSISTENT, er.ER_BATCH_PLAIN,
                                  er.ER_BATCH_PERSISTENT | er.ER_BATCH_HOST_OUT])
def test_batch_comp_equals_single_comp(ctx, mode):
    """The all-FP32 form of the batch: every job equals er_grid with
    ER_PREC_COMP, bit for bit."""
    import torch
    fws, ups = _batch_frameworks(ctx, n=8, seed=150)
    host = bool(mode & er.ER_BATCH_HOST_OUT)
    if host:
        outs = [torch.empty(f.dims, dtype=torch.float32, pin_memory=True) for f in fws]
    else:
        outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)],
                   mode | er.ER_BATCH_COMP)
    for u, f, o in zip(ups, fws, outs):
        single = ctx.grid(u, f.dims, precision=er.ER_PREC_COMP)
        assert np.array_equal(o.cpu().numpy(), single)


def test_rcp64_seed_error_bound(ctx):
    """The FP64 near terms of ER_PREC_NEAR64 refine the hardware reciprocal
    seed by one Newton step, which squares its relative error: the seed must
    stay below 2^-16 (so a refined reciprocal is within ~2^-32) over the
    squared distances the near pairs meet."""
    e0 = ctx.rcp64_seed_error()
    assert 0.0 < e0 < 2.0 ** -16, e0
