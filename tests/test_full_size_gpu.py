"""Parity at the workload sizes of the benchmarks, through properties that do
not need the oracle to evaluate everything: the full 256-framework batch and
the full 1e7-insertion Widom run sampled against the oracle at the same
points, a full-size (0.2 A) pocket-blocking grid bit-exact, and determinism."""
import numpy as np
import pytest

import emptyroom_b200 as er
import oracle
from conftest import grid_errors
from emptyroom_b200 import synth

pytestmark = pytest.mark.gpu


def _check(stats):
    assert stats["neg_ok"], stats
    assert stats["pos_ok"], stats
    assert stats["cap_ok"], stats


def test_full_batch_sampled_against_oracle(ctx):
    """All 256 config-2 frameworks in one persistent autotuned launch (the
    benchmark's step, default precision): per grid 48 points with E < -10 K
    (where the grid has them) and 16 uniform points against the FP64 oracle,
    at the strict bound (1e-5 relative below -10 K)."""
    import torch
    fws = synth.config2(n_frameworks=256, seed=1000)
    ups = ctx.upload_many([(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws])
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)],
                   er.ER_BATCH_PERSISTENT | er.ER_BATCH_AUTOTUNE)
    rng = np.random.default_rng(5)
    got, ref, S = [], [], []
    n_deep = 0
    for f, o in zip(fws, outs):
        flat = o.reshape(-1)
        deep = torch.nonzero(flat < -10.0).reshape(-1).cpu().numpy()
        idx = np.concatenate([rng.choice(deep, size=min(48, deep.size), replace=False),
                              rng.integers(0, flat.numel(), size=16)])
        pts = np.stack(np.unravel_index(idx, f.dims), -1) / (np.array(f.dims) - 1.0)
        e, s, _ = oracle.points_cells(f.particles(), f.t_matrix, f.rep, f.rc2, pts, 1e-12)
        got.append(flat[torch.from_numpy(idx).cuda()].cpu().numpy())
        ref.append(e)
        S.append(s)
        n_deep += int((e < -10.0).sum())
    st = grid_errors(np.concatenate(got), np.concatenate(ref), np.concatenate(S))
    _check(st)
    assert n_deep > 5000, st
    for u in ups:
        u.release()


def test_config3_cell_at_config1_density_full_grid(ctx):
    """The config-3 cell with 646 atoms (the config-1 number density, so it has
    pores) on the full 256^3 grid: every point of the default mode against the
    ER_PREC_FP64 grid (same pair set, FP64 terms and sums), which is pinned to
    the FP64 oracle on sampled points."""
    import torch
    f = synth.make_framework(3, (30.1, 32.4, 28.7), (85.0, 95.0, 110.0), 646, n_types=4,
                             probe="CH4", rc=12.5, d_min=1.2, name="config3_646")
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = (256, 256, 256)
    e = torch.empty(dims, dtype=torch.float32, device="cuda")
    e64 = torch.empty(dims, dtype=torch.float64, device="cuda")
    ctx.grid_device(fw, dims, e.data_ptr())
    ctx.grid_device(fw, dims, e64.data_ptr(), precision=er.ER_PREC_FP64, f64=True)
    ctx.synchronize()
    rng = np.random.default_rng(2)
    idx = rng.integers(0, 256, size=(2000, 3))
    ref, S, _ = oracle.points_cells(P, f.t_matrix, f.rep, f.rc2, idx / 255.0, 1e-12)
    pin = e64[idx[:, 0], idx[:, 1], idx[:, 2]].cpu().numpy()
    ok = ref < er.ER_ENERGY_CAP
    assert np.all(np.abs(pin[ok] - ref[ok]) <= 1e-12 * S[ok] + 1e-9)
    deep = e64 < -10.0
    assert int(deep.sum().item()) > 500000
    rel = ((e.double() - e64).abs() / e64.abs())[deep]
    assert float(rel.max().item()) <= 1e-5
    shallow = (e64 >= -10.0) & (e64 < 0)
    assert float((e.double() - e64).abs()[shallow].max().item()) <= 2e-3
    fw.release()


def test_full_widom_energies_sampled(ctx):
    """1e7 Philox insertions in a config-1 cell (Xe, 298 K): the energies of
    2000 sampled insertions against the oracle at the same points, and K_H
    consistent with the FP64 sum of the returned energies."""
    f = synth.make_framework(0, (25.8,) * 3, (90,) * 3, 424, probe="Xe")
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    n = 10_000_000
    r = ctx.henry(fw, 298.0, n, seed=3, want_energies=True)
    E = r["energies"]
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(n, size=2000, replace=False))
    pts = np.array([oracle.insertion_point(3, int(i)) for i in idx])
    ref = oracle.points(P, f.t_matrix, f.rep, f.rc2, pts, 1e-16)
    S = oracle.points_abs(P, f.t_matrix, f.rep, f.rc2, pts, 1e-16)
    _check(grid_errors(E[idx], ref, S))
    w = np.exp(-E.astype(np.float64) / 298.0)
    assert abs(w.sum() - r["sum_w"]) <= 1e-5 * r["sum_w"]


def test_full_size_henry_kh_with_device_mask(ctx):
    """A config-4 cell (Xe, 298 K) at the benchmark's size: 0.2 A grid ->
    device pocket mask -> 1e7 Philox insertions; K_H within 1e-6 of the FP64
    oracle (its own grid and flood fill, the same points, the cell-list sum of
    the reference's terms)."""
    import torch
    f = synth.config4(1, seed=4000)[0]
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    dims = f.dims
    g = torch.empty(dims, dtype=torch.float32, device="cuda")
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    ctx.grid_device(fw, dims, g.data_ptr())
    n_p = ctx.block_pockets_device(g.data_ptr(), dims, 298.0, m.data_ptr())
    n = 10_000_000
    r = ctx.henry_device_mask(fw, 298.0, n, 3, m.data_ptr(), dims)
    E = oracle.grid_cells(P, f.t_matrix, f.rep, f.rc2, dims)
    blocked, n_po, _ = oracle.block_pockets(E, 298.0)
    mask_o = ((blocked == 1e13) & (E != 1e13)).astype(np.uint8)
    assert n_p == n_po and n_p > 0
    assert np.array_equal(m.cpu().numpy(), mask_o)
    o = oracle.henry_cells(P, f.t_matrix, f.rep, f.rc2, 298.0, 3, n, mask=mask_o)
    assert r["n_blocked"] == o["n_blocked"] > 0
    assert abs(r["sum_w"] - o["sum_w"]) <= 1e-6 * o["sum_w"]
    kh_o = o["sum_w"] / n / 298.0 / 8.314
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= 1e-6 * kh_o
    fw.release()


def test_full_size_pockets_bit_exact(ctx):
    """A config-4 pocket-blocking grid (0.2 A, 129^3) from the GPU grid: the
    device mask and pocket count equal the oracle's flood fill."""
    import torch
    f = synth.config4(1, seed=4000)[0]
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    dims = f.dims
    g = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, g.data_ptr())
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    n_p = ctx.block_pockets_device(g.data_ptr(), dims, 298.0, m.data_ptr())
    E = g.cpu().numpy().astype(np.float64)
    ob, on, _ = oracle.block_pockets(E, 298.0)
    assert n_p == on
    assert np.array_equal(m.cpu().numpy(), ((ob == 1e13) & (E != 1e13)).astype(np.uint8))


def test_full_grid_deterministic(ctx):
    """Config-3 cell at 256^3: two launches give the same bits."""
    import torch
    f = synth.config3()
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    dims = (256, 256, 256)
    a = torch.empty(dims, dtype=torch.float32, device="cuda")
    b = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, a.data_ptr(), precision=er.ER_TILE_P8)
    ctx.grid_device(fw, dims, b.data_ptr(), precision=er.ER_TILE_P8)
    ctx.synchronize()
    assert torch.equal(a, b)
