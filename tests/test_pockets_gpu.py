"""GPU pocket blocking (er_block_pockets*) against the reference's
FindAndBlockPockets: bit-exact blocked grids, pocket counts and segment
numbering on the golden fixtures, on random grids, and on real energy grids."""
import numpy as np
import pytest

import oracle
from conftest import golden
from emptyroom_b200 import synth

pytestmark = pytest.mark.gpu

POCKET_CASES = ["pockets_a", "pockets_b", "pockets_perc", "pockets_perc_dense", "pockets_sparse"]


@pytest.mark.parametrize("name", POCKET_CASES)
def test_pockets_match_golden(ctx, name):
    g = golden(name)
    blocked, n, seg = ctx.block_pockets(g["grid"], float(g["T"]), want_segments=True)
    assert n == int(g["n_pockets"])
    assert np.array_equal(blocked, g["blocked"])
    _, _, oseg = oracle.block_pockets(g["grid"], float(g["T"]))
    assert np.array_equal(seg, oseg)


@pytest.mark.parametrize("seed", range(12))
def test_pockets_random_grids(ctx, seed):
    rng = np.random.default_rng(seed)
    dims = tuple(int(x) for x in rng.integers(2, 30, size=3))
    T = float(rng.uniform(50, 400))
    p_open = float(rng.uniform(0.05, 0.9))
    E = np.where(rng.random(dims) < p_open, -T, 16 * T) * rng.uniform(0.5, 1.5, size=dims)
    blocked, n = ctx.block_pockets(E, T)
    ob, on, _ = oracle.block_pockets(E, T)
    assert n == on and np.array_equal(blocked, ob)


def test_pockets_threshold_is_inclusive(ctx):
    T = 100.0
    E = np.full((4, 5, 6), 15.0 * T)  # E >= 15 T: inaccessible
    E[1:3, 1:3, 1:3] = np.nextafter(15.0 * T, 0)
    blocked, n = ctx.block_pockets(E, T)
    ob, on, _ = oracle.block_pockets(E, T)
    assert n == on == 1 and np.array_equal(blocked, ob)


def test_pockets_all_open_and_all_blocked(ctx):
    T = 300.0
    E = np.full((7, 6, 5), -T)
    blocked, n = ctx.block_pockets(E, T)
    assert n == 0 and np.array_equal(blocked, E)
    E2 = np.full((7, 6, 5), 100 * T)
    blocked2, n2 = ctx.block_pockets(E2, T)
    assert n2 == 0 and np.array_equal(blocked2, E2)


def test_pockets_on_energy_grid_and_device_mask(ctx):
    """A framework energy grid at 0.5 A: host form vs oracle, device form mask."""
    import torch
    f = synth.config1(2)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    dims = (52, 52, 52)
    T = 298.0
    d = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, d.data_ptr())
    ctx.synchronize()
    E = d.cpu().numpy().astype(np.float64)
    blocked, n = ctx.block_pockets(E, T)
    ob, on, _ = oracle.block_pockets(E, T)
    assert n == on and np.array_equal(blocked, ob)
    m = torch.empty(dims, dtype=torch.uint8, device="cuda")
    nd = ctx.block_pockets_device(d.data_ptr(), dims, T, m.data_ptr())
    assert nd == on
    want = (ob == 1e13) & (E != 1e13)
    assert np.array_equal(m.cpu().numpy().astype(bool), want)


def test_pockets_large_grid(ctx):
    rng = np.random.default_rng(5)
    dims = (130, 130, 130)
    T = 298.0
    E = np.where(rng.random(dims) < 0.33, -T, 20 * T)
    blocked, n = ctx.block_pockets(E, T)
    ob, on, _ = oracle.block_pockets(E, T)
    assert n == on and np.array_equal(blocked, ob)
