"""The reference's file formats (CPU only): loaders against the reference's own
loader results (golden), settings parsing, grid text byte-compatibility."""
import os
import sys

import numpy as np
import pytest

import emptyroom_b200 as er
from conftest import GOLDEN, golden
from emptyroom_b200 import files

sys.path.insert(0, GOLDEN)
from make_golden import write_fixture_tree  # noqa: E402


@pytest.fixture()
def tree(tmp_path):
    write_fixture_tree(str(tmp_path))
    return tmp_path


def test_structure_matches_reference_loader(tree):
    g = golden("loader_syn1")
    s = files.Structure(tree, "SYN1")
    assert s.n_atoms == 6
    assert (s.a, s.b, s.c) == (g["a"], g["b"], g["c"])
    assert (s.alpha, s.beta, s.gamma) == (g["alpha"], g["beta"], g["gamma"])
    assert s.volume == g["volume"] and s.density == g["density"]
    assert np.array_equal(s.t_matrix, g["t_matrix"])
    assert np.array_equal(s.inv_t_matrix, g["inv_t_matrix"])
    # fmod keeps negative coordinates negative (src/Framework.cc:58-60)
    assert np.array_equal(s.frac, g["frac"]) and s.frac.min() < 0
    assert s.labels == ["Zn", "O", "C", "H", "C", "O"]


def test_forcefield_matches_reference_loader(tree):
    g = golden("loader_syn1")
    f = files.Forcefield(tree, "SYNFF")
    assert np.array_equal(np.array(f.eps), g["ff_eps"])
    assert np.array_equal(np.array(f.sig), g["ff_sig"])
    assert f.find("Xe") == (221.0, 4.10)
    with pytest.raises(files.FileError):
        f.find("Ar")


def test_mixing_matches_rule(tree):
    s = files.Structure(tree, "SYN1")
    f = files.Forcefield(tree, "SYNFF")
    eg, sg = f.find("CH4")
    P = files.mix_particles(s, f, eg, sg)
    eps_f = np.array([f.find(lab)[0] for lab in s.labels])
    sig_f = np.array([f.find(lab)[1] for lab in s.labels])
    e, s2 = er.lorentz_berthelot(eps_f, sig_f, eg, sg)
    assert np.array_equal(P[:, 3], e) and np.array_equal(P[:, 4], s2)
    assert np.array_equal(P[:, :3], s.frac)


def test_loader_errors(tree):
    with pytest.raises(files.FileError) as ei:
        files.Structure(tree, "NOPE")
    assert "failed to import" in str(ei.value)
    with pytest.raises(files.FileError):
        files.Forcefield(tree, "NOPE")
    with open(os.path.join(tree, "data", "masses.def"), "w") as fh:
        fh.write("[atom] [mass]\nZn 65.38\n")
    with pytest.raises(files.FileError) as ei:
        files.Structure(tree, "SYN1")
    assert "not present" in str(ei.value)


def test_adsorbate_mw(tree):
    assert files.adsorbate_mw(tree, "CH4") == 16.04
    with pytest.raises(files.FileError):
        files.adsorbate_mw(tree, "Xe")


def test_uc_roundtrip_and_missing(tree):
    os.makedirs(os.path.join(tree, "data", "uc_replications"))
    with pytest.raises(files.FileError):
        files.read_uc(tree, "SYN1", "once")
    files.write_uc(tree, "SYN1", "once", (2, 1, 3))
    assert files.read_uc(tree, "SYN1", "once") == (2, 1, 3)
    open(os.path.join(tree, "data", "uc_replications", "EMPTY_once.uc"), "w").close()
    with pytest.raises(files.FileError) as ei:
        files.read_uc(tree, "EMPTY", "once")
    assert "Problem reading UC file" in str(ei.value)


SIM_INPUT = """Forcefield SYNFF other.def # store as .def

GridResolution 0.25 A
CutoffRadius 11.0 A
VoidFractionEnergyThreshold 0
GridOutputFormat cube # txt or cube

FeynmanHibbs 0 # "1" or "0"
Temperature 298 K

NumberOfInsertionsPerA3 50
NumberOfTrials 300000
verbosemode 0
"""


def test_settings_parse_like_reference(tmp_path):
    p = tmp_path / "simulation.input"
    p.write_text(SIM_INPUT)
    s = files.read_settings(p, files.ER_SETTINGS_GRID)
    assert s["forcefield"] == "SYNFF" and s["grid_resolution"] == 0.25
    assert s["r_cutoff_squared"] == 121.0 and s["grid_output_format"] == "cube"
    assert s["temperature"] == 298 and s["insertions_per_a3"] == 50 and s["verbose"] == 0
    h = files.read_settings(p, files.ER_SETTINGS_HENRY)
    assert h == s


def test_settings_defaults_and_missing(tmp_path):
    p = tmp_path / "simulation.input"
    p.write_text("Forcefield X\nGridResolution 0.5\n")
    s = files.read_settings(p, files.ER_SETTINGS_GRID)
    assert s["r_cutoff_squared"] == 12.5 * 12.5 and s["grid_output_format"] == "txt"
    with pytest.raises(files.FileError) as ei:
        files.read_settings(p, files.ER_SETTINGS_HENRY)
    assert "Missing Temperature" in str(ei.value)
    p.write_text("GridResolution 0.5\n")
    with pytest.raises(files.FileError) as ei:
        files.read_settings(p, files.ER_SETTINGS_GRID)
    assert "Missing Forcefield" in str(ei.value)
    with pytest.raises(files.FileError):
        files.read_settings(tmp_path / "none.input", files.ER_SETTINGS_GRID)


def _txt_serial(grid):
    nx, ny, nz = grid.shape
    out = [f"{nx} {ny} {nz}  = (N_x,N_y,N_z) grid points (grid is in fractional coords). "
           "Endpoints included.\n"]
    for i in range(nx):
        for j in range(ny):
            out.append("".join("% 13.6E " % float(v) for v in grid[i, j]) + "\n")
    return "".join(out)


@pytest.mark.parametrize("threads", [1, 3, 0])
def test_grid_txt_bytes_match_serial_printf(tmp_path, threads):
    rng = np.random.default_rng(threads)
    g = (rng.standard_normal((5, 7, 9)) * 10.0 ** rng.integers(-3, 8, size=(5, 7, 9))).astype(
        np.float32)
    g[0, 0, 0] = 1e30
    g[1, 2, 3] = 0.0
    g[2, 2, 2] = -0.0
    p = tmp_path / "g.txt"
    files.write_grid_txt(p, g, n_threads=threads)
    assert p.read_text() == _txt_serial(g)
    back = files.read_grid_txt(p)
    assert back.shape == g.shape
    np.testing.assert_allclose(back, g.astype(np.float64), rtol=1e-6)


def test_grid_cube_bytes_match_serial_printf(tmp_path):
    rng = np.random.default_rng(9)
    g = (rng.standard_normal((4, 3, 8)) * 1e3).astype(np.float32)
    t, _, _ = er.cell_matrices(12.0, 13.0, 14.0, 80, 95, 110)
    p = tmp_path / "g.cube"
    files.write_grid_cube(p, g, t, n_threads=2)
    nx, ny, nz = g.shape
    hdr = ["\nThis is a grid file.\n", "%d % 13.6f % 13.6f % 13.6f\n" % (0, 0.0, 0.0, 0.0),
           "%d % 13.6f % 13.6f % 13.6f\n" % (nx, t[0, 0] / (nx - 1), 0.0, 0.0),
           "%d % 13.6f % 13.6f % 13.6f\n" % (ny, t[0, 1] / (ny - 1), t[1, 1] / (ny - 1), 0.0),
           "%d % 13.6f % 13.6f % 13.6f\n" % (nz, t[0, 2] / (nz - 1), t[1, 2] / (nz - 1),
                                            t[2, 2] / (nz - 1))]
    body = []
    for i in range(nx):
        for j in range(ny):
            line = ""
            for k in range(nz):
                line += "% 13.6E " % (float(g[i, j, k]) * 8.314 / 1000)
                if (k + 1) % 6 == 0:
                    line += "\n"
            body.append(line + "\n")
    assert p.read_text() == "".join(hdr) + "".join(body)


def test_grid_reader_rejects_truncated(tmp_path):
    p = tmp_path / "g.txt"
    files.write_grid_txt(p, np.zeros((3, 3, 3), dtype=np.float32))
    lines = p.read_text().splitlines(True)
    (tmp_path / "t.txt").write_text("".join(lines[:-2]))
    with pytest.raises(files.FileError):
        files.read_grid_txt(tmp_path / "t.txt")
