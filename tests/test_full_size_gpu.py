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
    """All 256 config-2 frameworks in one persistent autotuned launch; 24
    sampled points per grid against the FP64 oracle."""
    import torch
    fws = synth.config2(n_frameworks=256, seed=1000)
    ups = ctx.upload_many([(f.particles(), f.t_matrix, f.rep, f.rc2) for f in fws])
    outs = [torch.empty(f.dims, dtype=torch.float32, device="cuda") for f in fws]
    ctx.grid_batch([(u, f.dims, o.data_ptr()) for u, f, o in zip(ups, fws, outs)],
                   er.ER_BATCH_PERSISTENT | er.ER_BATCH_AUTOTUNE)
    rng = np.random.default_rng(5)
    got, ref, S = [], [], []
    for f, o in zip(fws, outs):
        dims = np.array(f.dims)
        idx = rng.integers(0, dims, size=(24, 3))
        pts = idx / (dims - 1.0)
        e = o[idx[:, 0], idx[:, 1], idx[:, 2]].cpu().numpy()
        P = f.particles()
        got.append(e)
        ref.append(oracle.points(P, f.t_matrix, f.rep, f.rc2, pts, 1e-12))
        S.append(oracle.points_abs(P, f.t_matrix, f.rep, f.rc2, pts, 1e-12))
    _check(grid_errors(np.concatenate(got), np.concatenate(ref), np.concatenate(S)))
    for u in ups:
        u.release()


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
