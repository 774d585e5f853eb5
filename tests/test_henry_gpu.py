"""Parity of the CUDA Widom path (er_henry) with the FP64 oracle fed the same
Philox insertion points: K_H within 1e-6 relative, per-insertion energies
within the grid tolerances, blocked-insertion counts exact."""
import numpy as np
import pytest

import oracle
from conftest import grid_errors, rotated_cell
from emptyroom_b200 import synth

pytestmark = pytest.mark.gpu

KH_RTOL = 1e-6


def _fw(ctx, seed=0, n_atoms=424, probe="Xe"):
    f = synth.make_framework(seed, (25.8, 25.8, 25.8), (90, 90, 90), n_atoms, probe=probe)
    P = f.particles()
    return f, P, ctx.upload(P, f.t_matrix, f.rep, f.rc2)


def _kh(sum_w, n, T):
    return sum_w / n / T / 8.314


@pytest.mark.parametrize("seed,n_ins", [(0, 100000), (1, 37777), (2, 1), (3, 257)])
def test_henry_matches_oracle(ctx, seed, n_ins):
    f, P, fw = _fw(ctx, seed)
    T = 298.0
    r = ctx.henry(fw, T, n_ins, seed=seed + 10, want_energies=True)
    o = oracle.henry(P, f.t_matrix, f.rep, f.rc2, T, seed + 10, n_ins, want_energies=True)
    pts = np.array([oracle.insertion_point(seed + 10, i) for i in range(min(n_ins, 3000))])
    S = oracle.points_abs(P, f.t_matrix, f.rep, f.rc2, pts, 1e-16)
    st = grid_errors(r["energies"][:len(pts)], o["energies"][:len(pts)], S)
    assert st["neg_ok"] and st["pos_ok"] and st["cap_ok"], st
    kh_o = _kh(o["sum_w"], n_ins, T)
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= KH_RTOL * kh_o
    assert abs(r["sum_w"] - o["sum_w"]) <= KH_RTOL * o["sum_w"]
    if o["sum_w"] > 0:
        mean_o = o["sum_ew"] / o["sum_w"]
        assert abs(r["mean_energy"] - mean_o) <= 1e-5 * abs(mean_o) + 1e-3
    assert r["n_insertions"] == n_ins and r["n_blocked"] == 0


def test_henry_config1_points(ctx):
    """config-1 framework, 1e5 insertions at 298 K (CH4)."""
    f = synth.config1(0)
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    r = ctx.henry(fw, 298.0, 100000, seed=1234)
    o = oracle.henry(P, f.t_matrix, f.rep, f.rc2, 298.0, 1234, 100000)
    kh_o = _kh(o["sum_w"], 100000, 298.0)
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= KH_RTOL * kh_o


def test_henry_deterministic(ctx):
    f, P, fw = _fw(ctx, 4)
    a = ctx.henry(fw, 300.0, 50000, seed=9, want_energies=True)
    b = ctx.henry(fw, 300.0, 50000, seed=9, want_energies=True)
    assert np.array_equal(a["energies"], b["energies"]) and a["sum_w"] == b["sum_w"]
    c = ctx.henry(fw, 300.0, 50000, seed=10)
    assert c["sum_w"] != a["sum_w"]


def test_henry_energies_independent_of_bin_order(ctx):
    """A bin inside one warp's positions keeps the run-dependent order of its
    atomic slots; only each warp's set of insertions is fixed. Repeated calls
    (both points-per-thread paths) and six pipelines running the same
    framework and seed at once, their atomics racing one another, must give
    the same bits."""
    f = synth.config1(0)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    for n in (200_000, 2_000_000):
        ref = ctx.henry(fw, 298.0, n, seed=21, want_energies=True)
        for _ in range(2):
            r = ctx.henry(fw, 298.0, n, seed=21, want_energies=True)
            assert np.array_equal(r["energies"], ref["energies"])
        got, _ = ctx.henry_batch([fw] * 6, 298.0, n, [21] * 6)
        for g in got:
            assert g["sum_w"] == ref["sum_w"] and g["mean_energy"] == ref["mean_energy"]


@pytest.mark.parametrize("n_ins", [30000, 1_050_000])
def test_henry_triclinic_masked_matches_oracle(ctx, n_ins):
    """A small triclinic cell (85/100/115 degrees, images replicated along
    every axis) behind a pocket mask, through both points-per-thread paths:
    blocked counts exact, K_H within 1e-6 of the cell-list FP64 oracle, and
    (the smaller run) the energies of the first 3000 unblocked insertions
    within the grid tolerances."""
    f = synth.make_framework(77, (14.0, 16.0, 18.0), (85.0, 100.0, 115.0), 90, probe="CH4")
    P = f.particles()
    fw = ctx.upload(P, f.t_matrix, f.rep, f.rc2)
    rng = np.random.default_rng(5)
    mask = (rng.random((18, 20, 22)) < 0.05).astype(np.uint8)
    T = 298.0
    want = n_ins < 100000
    r = ctx.henry(fw, T, n_ins, seed=33, block_mask=mask, want_energies=want)
    o = oracle.henry_cells(P, f.t_matrix, f.rep, f.rc2, T, 33, n_ins, mask=mask,
                           want_energies=want)
    assert r["n_blocked"] == o["n_blocked"] > 0
    kh_o = _kh(o["sum_w"], n_ins, T)
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= KH_RTOL * kh_o
    if want:
        ok = np.flatnonzero(np.isfinite(o["energies"]))[:3000]
        assert np.array_equal(np.isinf(r["energies"]), np.isinf(o["energies"]))
        pts = np.array([oracle.insertion_point(33, int(i)) for i in ok])
        S = oracle.points_abs(P, f.t_matrix, f.rep, f.rc2, pts, 1e-16)
        st = grid_errors(r["energies"][ok], o["energies"][ok], S)
        assert st["neg_ok"] and st["pos_ok"] and st["cap_ok"], st


@pytest.mark.parametrize("n_ins", [40000, 1_050_000])
def test_henry_rotated_cell_matches_oracle(ctx, n_ins):
    """A cell matrix that is not upper triangular: the insertion points go to
    Cartesian coordinates through the positioning frame, the exact cutoff
    decisions through the cell matrix itself. K_H within 1e-6 and (the
    smaller run) the first 3000 energies within the grid tolerances of the
    FP64 oracle on the same rotated matrix."""
    f = synth.make_framework(160, (16.0, 19.0, 17.5), (75, 105, 98), 140, probe="Kr")
    P = f.particles()
    t = rotated_cell(f.t_matrix, 3)
    assert abs(t[1, 0]) > 1e-3 and abs(t[2, 0]) > 1e-3
    fw = ctx.upload(P, t, f.rep, f.rc2)
    T = 298.0
    want = n_ins < 100000
    r = ctx.henry(fw, T, n_ins, seed=44, want_energies=want)
    o = oracle.henry_cells(P, t, f.rep, f.rc2, T, 44, n_ins, want_energies=want)
    kh_o = _kh(o["sum_w"], n_ins, T)
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= KH_RTOL * kh_o
    if want:
        pts = np.array([oracle.insertion_point(44, i) for i in range(3000)])
        S = oracle.points_abs(P, t, f.rep, f.rc2, pts, 1e-16)
        st = grid_errors(r["energies"][:3000], o["energies"][:3000], S)
        assert st["neg_ok"] and st["pos_ok"] and st["cap_ok"], st


def test_henry_with_block_mask(ctx):
    f, P, fw = _fw(ctx, 5, n_atoms=300)
    T = 298.0
    dims = (24, 24, 24)
    g = ctx.grid(fw, dims).astype(np.float64)
    rng = np.random.default_rng(0)
    mask = (rng.random(dims) < 0.02).astype(np.uint8)
    n = 60000
    r = ctx.henry(fw, T, n, seed=77, block_mask=mask, want_energies=True)
    o = oracle.henry(P, f.t_matrix, f.rep, f.rc2, T, 77, n, mask=mask, want_energies=True)
    assert r["n_blocked"] == o["n_blocked"] > 0
    blocked = np.isinf(o["energies"])
    assert np.array_equal(np.isinf(r["energies"]), blocked)
    kh_o = _kh(o["sum_w"], n, T)
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= KH_RTOL * kh_o
    del g


def test_henry_all_blocked(ctx):
    f, P, fw = _fw(ctx, 6, n_atoms=50)
    mask = np.ones((4, 4, 4), dtype=np.uint8)
    r = ctx.henry(fw, 298.0, 5000, seed=1, block_mask=mask)
    assert r["n_blocked"] == 5000 and r["sum_w"] == 0.0 and r["kh_mol_m3_pa"] == 0.0


def test_henry_lse_form_consistent(ctx):
    f, P, fw = _fw(ctx, 7)
    r = ctx.henry(fw, 150.0, 20000, seed=3)
    assert np.isclose(r["sum_w"], r["sum_w_scaled"] * np.exp(r["log_scale"]), rtol=1e-14)
    assert np.isclose(r["mean_energy"], r["sum_ew_scaled"] / r["sum_w_scaled"], rtol=1e-14)


def test_henry_invalid(ctx):
    import emptyroom_b200 as er
    f, P, fw = _fw(ctx, 8, n_atoms=20)
    with pytest.raises(er.ErError):
        ctx.henry(fw, -1.0, 100, seed=0)
    with pytest.raises(er.ErError):
        ctx.henry(fw, 298.0, 0, seed=0)


def test_henry_device_mask_pipeline(ctx):
    """grid -> device pocket mask -> Widom with that mask, against the oracle
    pipeline on the same grid."""
    import torch
    f, P, fw = _fw(ctx, 12, n_atoms=424)
    T = 298.0
    dims = (40, 40, 40)
    g = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, g.data_ptr())
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    n_p = ctx.block_pockets_device(g.data_ptr(), dims, T, m.data_ptr())
    E = g.cpu().numpy().astype(np.float64)
    ob, on, _ = oracle.block_pockets(E, T)
    assert n_p == on
    mask = ((ob == 1e13) & (E != 1e13)).astype(np.uint8)
    assert np.array_equal(m.cpu().numpy(), mask)
    n = 50000
    r = ctx.henry_device_mask(fw, T, n, 21, m.data_ptr(), dims)
    o = oracle.henry(P, f.t_matrix, f.rep, f.rc2, T, 21, n, mask=mask)
    assert r["n_blocked"] == o["n_blocked"]
    kh_o = _kh(o["sum_w"], n, T)
    assert abs(r["kh_mol_m3_pa"] - kh_o) <= KH_RTOL * kh_o


def _sequential(ctx, fws, T, n, seeds, dims):
    """The single-call pipeline: er_grid (device) -> er_block_pockets_device
    -> er_henry with the device mask; or er_henry alone."""
    import torch
    out, pockets = [], []
    for fw, s in zip(fws, seeds):
        if dims is None:
            out.append(ctx.henry(fw, T, n, s))
            pockets.append(0)
            continue
        g = torch.empty(dims, dtype=torch.float32, device="cuda")
        m = torch.empty(dims, dtype=torch.uint8, device="cuda")
        ctx.grid_device(fw, dims, g.data_ptr())
        pockets.append(ctx.block_pockets_device(g.data_ptr(), dims, T, m.data_ptr()))
        out.append(ctx.henry_device_mask(fw, T, n, s, m.data_ptr(), dims))
    return out, pockets


@pytest.mark.parametrize("dims", [None, (33, 33, 33)])
def test_henry_batch_equals_single_calls(ctx, dims):
    """er_henry_batch runs frameworks on concurrent pipelines; every entry
    must equal the single calls bit for bit (seven frameworks of different
    sizes, more than there are pipelines), twice in a row."""
    T = 298.0
    fws = []
    for k, na in enumerate([424, 120, 800, 50, 424, 300, 610]):
        f = synth.make_framework(40 + k, (25.8, 25.8, 25.8), (90, 90, 90), na, probe="Xe")
        fws.append(ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2))
    seeds = [7 + 3 * k for k in range(len(fws))]
    n = 60000
    ref, ref_p = _sequential(ctx, fws, T, n, seeds, dims)
    for _ in range(2):
        got, got_p = ctx.henry_batch(fws, T, n, seeds, block_dims=dims)
        assert got_p == ref_p
        for a, b in zip(got, ref):
            assert a == b
    if dims is not None:
        assert sum(ref_p) > 0 and any(r["n_blocked"] > 0 for r in ref)


def test_henry_batch_errors(ctx):
    import emptyroom_b200 as er
    f, P, fw = _fw(ctx, 3, n_atoms=100)
    assert ctx.henry_batch([], 298.0, 100, []) == ([], [])
    with pytest.raises(er.ErError):
        ctx.henry_batch([fw], -1.0, 100, [1])
    with pytest.raises(er.ErError):
        ctx.henry_batch([fw], 298.0, 100, [1], block_dims=(1, 8, 8))

    class Gone:
        id = 987654
    with pytest.raises(er.ErError, match="entry 1"):
        ctx.henry_batch([fw, Gone()], 298.0, 100, [1, 2])
    # the context stays usable
    assert ctx.henry_batch([fw], 298.0, 1000, [5])[0][0] == ctx.henry(fw, 298.0, 1000, 5)


def test_henry_stage_timing(ctx):
    """er_ctx_set_timing / er_henry_last_timing: per-stage device times of the
    last er_henry call, positive and within the call's own duration; timing
    leaves the result unchanged and is an error while it is off."""
    import time

    import emptyroom_b200 as er
    f, P, fw = _fw(ctx, 4, n_atoms=300)
    ref = ctx.henry(fw, 298.0, 200000, seed=9)
    ctx.set_timing(True)
    try:
        t0 = time.perf_counter()
        got = ctx.henry(fw, 298.0, 200000, seed=9)
        wall_ms = (time.perf_counter() - t0) * 1e3
        t = ctx.henry_timing()
    finally:
        ctx.set_timing(False)
    assert got == ref
    assert all(v > 0 for v in t.values()), t
    assert sum(t.values()) <= wall_ms, (t, wall_ms)
    with pytest.raises(er.ErError, match="timing is off"):
        ctx.henry_timing()


def test_blocked_insertions_match_the_reference_lookup(ctx):
    """2e6 Philox insertions against a sparse mask on a 23^3 grid: the blocked
    count equals the reference's lookup (src/gcmc.cc:155-157: cell
    floor(x / (1/(N-1))) clamped to N-2, any of its 8 corners blocked),
    evaluated here in numpy on the same points, including the points whose
    scaled coordinate lies within 1e-6 of a cell plane, where the library
    decides by the FP64 division itself."""
    f, P, fw = _fw(ctx, 7, n_atoms=60)
    N, n, seed = 23, 2_000_000, 17
    rng = np.random.default_rng(9)
    mask = (rng.random((N, N, N)) < 0.04).astype(np.uint8)
    r = ctx.henry(fw, 298.0, n, seed=seed, block_mask=mask)
    pts = oracle.insertion_points(seed, n)
    d = 1.0 / (N - 1)
    cell = np.minimum(np.floor(pts / d).astype(np.int64), N - 2)
    blocked = np.zeros(n, dtype=bool)
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                blocked |= mask[cell[:, 0] + di, cell[:, 1] + dj, cell[:, 2] + dk] != 0
    q = pts * (N - 1)
    assert int((np.abs(q - np.rint(q)) < 1e-6).sum()) > 0  # the division path is met
    assert r["n_blocked"] == int(blocked.sum())
