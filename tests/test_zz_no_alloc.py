"""er_henry_stats_noalloc, the entry point for callers that cannot allocate
device memory (a code that owns all of its device memory through its own
pool, or a loop that cannot take cudaMalloc's implicit synchronisation).
It reduces energies the caller holds on the device using only a static
device array, and must give er_henry's statistics for the same energies.
This file is collected last; each test builds its own inputs."""
import ctypes

import numpy as np
import pytest

from emptyroom_b200 import _capi, synth
from emptyroom_b200._capi import ErHenryResult

pytestmark = pytest.mark.gpu

KH_RTOL = 1e-6  # the K_H tolerance of the Widom parity tests


def _noalloc(ctx, energies_dev, n, T):
    out = ErHenryResult()
    st = _capi.lib().er_henry_stats_noalloc(ctx.handle, ctypes.c_void_p(energies_dev), int(n),
                                            float(T), ctypes.byref(out))
    return st, out


def _close(a, b):
    return abs(a - b) <= KH_RTOL * abs(b)


def test_noalloc_stats_match_er_henry_on_two_calls(ctx):
    import torch
    f = synth.make_framework(41, (25.8, 25.8, 25.8), (90, 90, 90), 300, probe="Xe")
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    T = 298.0
    rng = np.random.default_rng(3)
    mask = (rng.random((20, 20, 20)) < 0.03).astype(np.uint8)
    runs = [ctx.henry(fw, T, 200000, seed=5, block_mask=mask, want_energies=True),
            ctx.henry(fw, T, 70001, seed=6, want_energies=True)]
    for ref in runs:  # two calls in a row, different sizes, the static array reused
        E = torch.from_numpy(ref["energies"]).cuda()
        st, got = _noalloc(ctx, E.data_ptr(), E.numel(), T)
        assert st == 0, _capi.lib().er_ctx_last_error(ctx.handle)
        assert _close(got.kh_mol_m3_pa, ref["kh_mol_m3_pa"])
        assert _close(got.sum_w, ref["sum_w"])
        assert _close(got.mean_energy, ref["mean_energy"])
        assert got.n_insertions == ref["n_insertions"]
        assert got.n_blocked == ref["n_blocked"]
    assert runs[0]["n_blocked"] > 0
    fw.release()


def test_noalloc_rejects_out_of_range_sizes(ctx):
    import torch
    E = torch.zeros(16, dtype=torch.float32, device="cuda")
    st, _ = _noalloc(ctx, E.data_ptr(), 0, 298.0)
    assert st == 7  # ER_ERR_LIMIT
    st, _ = _noalloc(ctx, E.data_ptr(), (1 << 31), 298.0)
    assert st == 7
    assert b"ER_HENRY_STATS_NOALLOC_MAX_N" in _capi.lib().er_ctx_last_error(ctx.handle)


def test_noalloc_blocked_and_undefined_energies(ctx):
    """+inf entries (blocked insertions) have weight 0 and are counted; a NaN
    or -inf entry has no defined Boltzmann weight and fails the call."""
    import torch
    T = 298.0
    e = np.full(1000, -500.0, dtype=np.float32)
    e[::7] = np.inf
    E = torch.from_numpy(e).cuda()
    st, got = _noalloc(ctx, E.data_ptr(), e.size, T)
    assert st == 0
    n_inf = int(np.isinf(e).sum())
    assert got.n_blocked == n_inf
    kh = (e.size - n_inf) * np.exp(500.0 / T) / e.size / T / 8.314
    assert _close(got.kh_mol_m3_pa, kh)
    for bad in (np.nan, -np.inf):
        e2 = e.copy()
        e2[3] = bad
        E2 = torch.from_numpy(e2).cuda()
        st, _ = _noalloc(ctx, E2.data_ptr(), e2.size, T)
        assert st == 1  # ER_ERR_INVALID
        assert b"NaN or -inf" in _capi.lib().er_ctx_last_error(ctx.handle)


def test_noalloc_at_the_documented_maximum(ctx):
    """n = ER_HENRY_STATS_NOALLOC_MAX_N (2^31 - 1 energies, 8.6 GB): with a
    constant energy c every weight is exp(-c/T), so K_H = exp(-c/T)/(T 8.314)
    and <E> = c in closed form; the block partition must not overflow."""
    import torch
    n = _capi.ER_HENRY_STATS_NOALLOC_MAX_N
    c, T = -1234.5, 298.0
    E = torch.full((n,), c, dtype=torch.float32, device="cuda")
    # the fill runs on torch's stream, the library on its own non-blocking one
    torch.cuda.synchronize()
    try:
        st, got = _noalloc(ctx, E.data_ptr(), n, T)
        assert st == 0, _capi.lib().er_ctx_last_error(ctx.handle)
        assert got.n_insertions == n and got.n_blocked == 0
        kh = np.exp(-c / T) / T / 8.314
        assert abs(got.kh_mol_m3_pa - kh) <= 1e-12 * kh
        assert got.mean_energy == c
        st, _ = _noalloc(ctx, E.data_ptr(), n + 1, T)
        assert st == 7  # ER_ERR_LIMIT
    finally:
        del E
        torch.cuda.empty_cache()
