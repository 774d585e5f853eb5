"""C-ABI library checks that need no GPU: exports, host helpers, error paths."""
import ctypes
import os
import re

import numpy as np
import pytest

import emptyroom_b200 as er
from emptyroom_b200 import _capi
from conftest import ROOT, golden

HEADER = os.path.join(ROOT, "include", "emptyroom_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(er_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_bindings_cover_header():
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_status_strings():
    L = _capi.lib()
    assert L.er_status_string(0) == b"ok"
    assert L.er_status_string(7) == b"size limit exceeded"
    assert b"sm_100a" in L.er_version()


def test_cell_matrices_match_reference_loader():
    g = golden("loader_syn1")
    t, inv, vol = er.cell_matrices(float(g["a"]), float(g["b"]), float(g["c"]),
                                   float(g["alpha"]) * 180 / np.pi, float(g["beta"]) * 180 / np.pi,
                                   float(g["gamma"]) * 180 / np.pi)
    np.testing.assert_allclose(t, g["t_matrix"], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(inv, g["inv_t_matrix"], rtol=1e-13, atol=1e-15)
    assert abs(vol - float(g["volume"])) <= 1e-10 * vol
    np.testing.assert_allclose(t @ inv, np.eye(3), atol=1e-13)


def test_degenerate_cell_rejected():
    with pytest.raises(er.ErError):
        er.cell_matrices(10, 10, 10, 60, 60, 180)


@pytest.mark.parametrize("seed", range(5))
def test_replication_factors_cover_every_image(seed):
    """With rep = floor(rc / w) + 1 no image beyond rep is within rc of any grid point."""
    import oracle
    from emptyroom_b200 import synth
    rng = np.random.default_rng(seed)
    abc = rng.uniform(7, 14, size=3)
    ang = rng.uniform(70, 110, size=3)
    fw = synth.make_framework(seed, abc, ang, 12, probe="Kr", rc=float(rng.uniform(6, 11)))
    P = fw.particles()
    rep = np.array(fw.rep)
    dims = (5, 4, 6)
    g1 = oracle.grid(P, fw.t_matrix, rep, fw.rc2, dims)
    g2 = oracle.grid(P, fw.t_matrix, rep + 1, fw.rc2, dims)
    np.testing.assert_allclose(g1, g2, rtol=1e-12, atol=1e-9)


def test_synth_positions_respect_min_distance():
    t, _, _ = er.cell_matrices(12.0, 13.0, 11.0, 80.0, 95.0, 105.0)
    f = er.synth_positions(5, t, 150, 1.2)
    assert f.shape == (150, 3) and f.min() >= 0 and f.max() < 1
    d = f[:, None, :] - f[None, :, :]
    d -= np.floor(d + 0.5)
    best = np.full(d.shape[:2], np.inf)
    for sh in np.array(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1])).T.reshape(-1, 3):
        c = (d + sh) @ t.T
        best = np.minimum(best, (c ** 2).sum(-1))
    np.fill_diagonal(best, np.inf)
    assert np.sqrt(best.min()) >= 1.2
    # deterministic
    assert np.array_equal(f, er.synth_positions(5, t, 150, 1.2))


def test_synth_positions_density_limit():
    t, _, _ = er.cell_matrices(8.0, 8.0, 8.0, 90, 90, 90)
    with pytest.raises(er.ErError):
        er.synth_positions(1, t, 2000, 1.2)


def test_host_philox_and_points_match_oracle():
    import oracle
    for ctr, key in [((1, 2, 3, 4), (5, 6)), ((0xdeadbeef, 0, 7, 1 << 31), (99, 12345))]:
        assert np.array_equal(er.philox4x32_10(ctr, key), oracle.philox4x32_10(ctr, key))
    for i in [0, 1, 2, 1 << 33, 123456789]:
        assert np.array_equal(er.insertion_point(42, i), oracle.insertion_point(42, i))


def test_ctx_create_without_gpu_reports_cuda_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert _capi.lib().er_ctx_create(0, ctypes.byref(h)) == 2  # ER_ERR_CUDA
    assert not h.value


def test_lorentz_berthelot_matches_reference_rule():
    e, s2 = er.lorentz_berthelot([30.0, 52.83], [3.12, 3.43], 148.0, 3.73)
    np.testing.assert_allclose(e, np.sqrt(148.0 * np.array([30.0, 52.83])), rtol=0)
    np.testing.assert_allclose(s2, ((3.73 + np.array([3.12, 3.43])) / 2.0) ** 2, rtol=0)


def test_noalloc_limit_matches_header():
    import re
    hdr = open(os.path.join(ROOT, "include", "emptyroom_b200.h")).read()
    m = re.search(r"#define ER_HENRY_STATS_NOALLOC_MAX_N (\d+)LL", hdr)
    assert m and int(m.group(1)) == _capi.ER_HENRY_STATS_NOALLOC_MAX_N == 2**31 - 1
