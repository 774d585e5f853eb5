"""Pins the CPU oracle (oracle/er_oracle.c) to the reference's own code.

Two anchors: the golden fixtures in tests/golden (outputs of the reference's
src/computegridsheet.h, src/pocketblocking.cc, src/Framework.cc and
src/Forcefield.cc, produced by tests/golden/make_golden.py), and, where
oracle/_ref/libref.so is present, the reference code run live on fresh
seeded inputs. CPU only.
"""
import numpy as np
import pytest

import oracle
from conftest import golden

GRID_CASES = ["grid_cubic", "grid_triclinic", "grid_rep2"]
POCKET_CASES = ["pockets_a", "pockets_b", "pockets_perc", "pockets_perc_dense", "pockets_sparse"]


@pytest.mark.parametrize("name", GRID_CASES)
def test_oracle_grid_matches_golden_bitwise(name):
    g = golden(name)
    e = oracle.grid(g["particles"], g["t_matrix"], g["rep"], float(g["rc2"]), g["dims"])
    assert np.array_equal(e, g["grid"])


@pytest.mark.parametrize("name", GRID_CASES)
def test_oracle_accessibility_matches_golden(name):
    g = golden(name)
    a = oracle.accessibility(g["particles"], g["t_matrix"], g["dims"])
    assert np.array_equal(a, g["accessibility"])


@pytest.mark.parametrize("name", GRID_CASES)
def test_oracle_points_equal_grid(name):
    """The point form (used for Widom) evaluates the same sum as the grid form."""
    g = golden(name)
    nx, ny, nz = (int(x) for x in g["dims"])
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = np.stack([ii / (nx - 1), jj / (ny - 1), kk / (nz - 1)], axis=-1).reshape(-1, 3)
    e = oracle.points(g["particles"], g["t_matrix"], g["rep"], float(g["rc2"]), pts, 1e-12)
    assert np.array_equal(e.reshape(nx, ny, nz), g["grid"])


@pytest.mark.parametrize("name", POCKET_CASES)
def test_oracle_pockets_match_golden_bitwise(name):
    g = golden(name)
    blocked, n, seg = oracle.block_pockets(g["grid"], float(g["T"]))
    assert n == int(g["n_pockets"])
    assert np.array_equal(blocked, g["blocked"])
    # segment ids: -1 exactly where E >= 15 T, and numbered in scan order
    assert np.array_equal(seg < 0, g["grid"] >= 15.0 * float(g["T"]))
    first = {}
    for idx, s in enumerate(seg.ravel()):
        if s >= 0 and s not in first:
            first[s] = idx
    assert list(first) == sorted(first)


def test_philox_known_answers():
    """Random123 known-answer vectors of Philox4x32-10 (Salmon et al., SC'11)."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        assert [int(x) for x in oracle.philox4x32_10(ctr, key)] == list(want)


def test_insertion_points_uniform():
    pts = np.array([oracle.insertion_point(7, i) for i in range(4000)])
    assert pts.min() >= 0.0 and pts.max() < 1.0
    assert np.all(np.abs(pts.mean(axis=0) - 0.5) < 0.02)
    assert len(np.unique(pts[:, 0])) == len(pts)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [101, 102])
def test_oracle_grid_matches_reference_live(seed):
    from emptyroom_b200 import synth
    fw = synth.make_framework(seed, (11.0 + seed % 3, 12.5, 10.0), (82.0, 97.0, 104.0), 30,
                              probe="Kr", rc=10.0)
    P = fw.particles()
    dims = (7, 6, 8)
    assert np.array_equal(oracle.grid(P, fw.t_matrix, fw.rep, fw.rc2, dims),
                          oracle.ref_grid(P, fw.t_matrix, fw.rep, fw.rc2, dims))
    assert np.array_equal(oracle.accessibility(P, fw.t_matrix, dims),
                          oracle.ref_accessibility(P, fw.t_matrix, dims))


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed,p", [(201, 0.25), (202, 0.32), (203, 0.5)])
def test_oracle_pockets_match_reference_live(seed, p):
    rng = np.random.default_rng(seed)
    T = 250.0
    E = np.where(rng.random((13, 11, 12)) < p, -T, 20 * T)
    b1, n1, _ = oracle.block_pockets(E, T)
    b2, n2 = oracle.ref_block_pockets(E, T)
    assert n1 == n2 and np.array_equal(b1, b2)


def test_oracle_interp_matches_golden_bitwise():
    """GCMC lookup restatement vs the reference's GuestFrameworkEnergy
    (src/gcmc.cc:145-177) on the golden grid and points."""
    g = golden("gcmc_interp")
    assert np.array_equal(oracle.grid_interp(g["grid"], g["pts"]), g["energy"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built here")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_interp_matches_reference_live(seed):
    rng = np.random.default_rng(seed)
    dims = tuple(int(x) for x in rng.integers(2, 30, size=3))
    grid = rng.normal(size=dims) * 100.0
    grid[rng.random(dims) < 0.05] = 1e13
    pts = rng.uniform(-3.0, 4.0, size=(3000, 3))
    assert np.array_equal(oracle.grid_interp(grid, pts), oracle.ref_grid_interp(grid, pts))


# ---------------------------------------------------------- cell-list form
def _cases():
    from emptyroom_b200 import synth
    return [synth.config1(0),
            synth.make_framework(61, (9.1, 11.3, 8.7), (72, 104, 97), 60, probe="Xe"),
            synth.make_framework(62, (21.0, 17.5, 26.0), (95, 80, 110), 700, probe="Kr")]


@pytest.mark.parametrize("k", range(3))
def test_cell_list_sum_equals_image_loop(k):
    """er_oracle_cells.c sums the same terms as the image loop: identical term
    counts, energies within a few ulps of sum |term| (only the order of the
    additions differs)."""
    f = _cases()[k]
    P = f.particles()
    pts = np.random.default_rng(k).random((400, 3))
    for min_r in (1e-12, 1e-16):
        e, s, c = oracle.points_cells(P, f.t_matrix, f.rep, f.rc2, pts, min_r)
        ref = oracle.points(P, f.t_matrix, f.rep, f.rc2, pts, min_r)
        S = oracle.points_abs(P, f.t_matrix, f.rep, f.rc2, pts, min_r)
        assert np.array_equal(c, oracle.points_pairs(P, f.t_matrix, f.rep, f.rc2, pts, min_r))
        assert np.all(np.abs(e - ref) <= 1e-13 * S)
        assert np.all(np.abs(s - S) <= 1e-13 * S)
    dims = (7, 6, 9)
    g = oracle.grid_cells(P, f.t_matrix, f.rep, f.rc2, dims)
    g0 = oracle.grid(P, f.t_matrix, f.rep, f.rc2, dims)
    S = oracle.grid_abs(P, f.t_matrix, f.rep, f.rc2, dims)
    assert np.all(np.abs(g - g0) <= 1e-13 * S)


@pytest.mark.parametrize("cell", ["cubic", "triclinic", "rotated"])
def test_cell_list_henry_equals_image_loop(cell):
    """The cell-list Widom oracle (the reference for the GPU Widom tests on
    triclinic and rotated cells) equals the image loop."""
    from conftest import rotated_cell
    from emptyroom_b200 import synth
    if cell == "cubic":
        f = synth.make_framework(63, (14.0, 15.0, 13.0), (90, 90, 90), 120, probe="Xe")
    elif cell == "triclinic":
        f = synth.make_framework(77, (14.0, 16.0, 18.0), (85.0, 100.0, 115.0), 90, probe="CH4")
    else:
        f = synth.make_framework(160, (16.0, 19.0, 17.5), (75, 105, 98), 140, probe="Kr")
    t = rotated_cell(f.t_matrix, 3) if cell == "rotated" else f.t_matrix
    P = f.particles()
    mask = (np.random.default_rng(2).random((9, 8, 10)) < 0.05).astype(np.uint8)
    for m in (None, mask):
        a = oracle.henry(P, t, f.rep, f.rc2, 298.0, 9, 3000, mask=m, want_energies=True)
        b = oracle.henry_cells(P, t, f.rep, f.rc2, 298.0, 9, 3000, mask=m,
                               want_energies=True)
        assert a["n_blocked"] == b["n_blocked"]
        assert abs(a["sum_w"] - b["sum_w"]) <= 1e-12 * a["sum_w"]
        fin = np.isfinite(a["energies"])
        assert np.array_equal(fin, np.isfinite(b["energies"]))


def test_workload_generators_equal_the_library():
    """The reference arm's frameworks (oracle/workloads.py) are the GPU arm's
    (emptyroom_b200/synth.py) bit for bit."""
    from emptyroom_b200 import synth
    from oracle import workloads
    for a, b in ((workloads.config2(256), synth.config2(256)),
                 (workloads.config4(8), synth.config4(8))):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            assert np.array_equal(x.particles(), y.particles())
            assert np.array_equal(x.t_matrix, y.t_matrix)
            assert tuple(x.rep) == tuple(y.rep) and tuple(x.dims) == tuple(y.dims)
