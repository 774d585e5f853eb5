"""GCMC grid lookup on the device (er_grid_interp) against the reference's
GuestFrameworkEnergy (golden fixture) and the oracle restatement: bit for bit,
FP64 and FP32 grids, host and device points."""
import numpy as np
import pytest

import emptyroom_b200 as er
import oracle
from conftest import golden
from emptyroom_b200 import synth

pytestmark = pytest.mark.gpu


def test_interp_matches_golden_bitwise(ctx):
    import torch
    g = golden("gcmc_interp")
    grid = torch.from_numpy(g["grid"]).cuda()
    e = ctx.grid_interp(grid.data_ptr(), g["grid"].shape, g["pts"], f64=True)
    assert np.array_equal(e, g["energy"])


def test_interp_on_float_grid_from_er_grid(ctx):
    """A grid written by er_grid (FP32, device) looked up at GCMC guest
    positions, device points and results."""
    import torch
    f = synth.config1(5)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    dims = (33, 29, 31)
    grid = torch.empty(dims, dtype=torch.float32, device="cuda")
    ctx.grid_device(fw, dims, grid.data_ptr())
    rng = np.random.default_rng(9)
    pts = rng.uniform(-1.0, 2.0, size=(100000, 3))
    d_pts = torch.from_numpy(pts).cuda()
    d_out = torch.empty(len(pts), dtype=torch.float64, device="cuda")
    ctx.grid_interp_device(grid.data_ptr(), dims, d_pts.data_ptr(), len(pts), d_out.data_ptr())
    ctx.synchronize()
    want = oracle.grid_interp(grid.cpu().numpy().astype(np.float64), pts)
    assert np.array_equal(d_out.cpu().numpy(), want)
    # host points give the same
    assert np.array_equal(ctx.grid_interp(grid.data_ptr(), dims, pts[:5000]), want[:5000])


def test_interp_rejects_bad_arguments(ctx):
    import torch
    g = np.zeros((4, 4, 4))
    pts = np.zeros((3, 3))
    with pytest.raises(er.ErError):  # grid in host memory
        ctx.grid_interp(g.ctypes.data, g.shape, pts, f64=True)
    d = torch.zeros((4, 4, 1), dtype=torch.float64, device="cuda")
    with pytest.raises(er.ErError):  # N < 2
        ctx.grid_interp(d.data_ptr(), (4, 4, 1), pts, f64=True)
