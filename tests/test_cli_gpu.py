"""The drop-in tools `writegrid` and `henry` (emptyroom_b200/bin) on a project
tree in the reference's layout: grid files against the FP64 oracle and
against the reference's own writegrid (compiled for sm_100a from its
sources, oracle/_ref/writegrid) run on the same tree; .out reports line by
line; henry's K_H against the reference's henry within statistical error."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT, grid_errors
from emptyroom_b200 import synth
from fixture_tree import particles_from_tree, read_out, write_tree

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "emptyroom_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def _run(exe, root, *args):
    r = subprocess.run([exe, *args], cwd=root, capture_output=True, text=True, timeout=600)
    return r


@pytest.fixture()
def tree(tmp_path):
    fw = synth.make_framework(31, (21.3, 19.7, 23.1), (82.0, 97.0, 104.0), 160, n_types=4,
                              probe="CH4", rc=12.5)
    name, ads = write_tree(str(tmp_path), fw, resolution=0.7)
    return tmp_path, name, ads


def test_writegrid_usage_and_errors(tmp_path):
    r = _run(os.path.join(BIN, "writegrid"), str(tmp_path))
    assert r.returncode != 0 and "Run as:" in r.stdout
    r = _run(os.path.join(BIN, "writegrid"), str(tmp_path), "A", "B")
    assert r.returncode != 0 and "masses.def" in r.stdout


def test_writegrid_matches_oracle(tree):
    root, name, ads = tree
    r = _run(os.path.join(BIN, "writegrid"), str(root), name, ads)
    assert r.returncode == 0, r.stdout + r.stderr
    from emptyroom_b200 import files
    g = files.read_grid_txt(os.path.join(root, "data", "grids", f"{name}_{ads}_SYNFF.txt"))
    s, P, rep = particles_from_tree(str(root), name, "SYNFF", ads)
    ref = oracle.grid(P, s.t_matrix, rep, 12.5 * 12.5, g.shape)
    S = oracle.grid_abs(P, s.t_matrix, rep, 12.5 * 12.5, g.shape)
    # the text holds 7 significant digits: add half a unit of the last one
    st = grid_errors(g, ref, S + 1e-6 * np.abs(ref) / 2e-6)
    assert st["neg_ok"] and st["pos_ok"], st
    assert g.shape == tuple(int(np.ceil(L / 0.7)) for L in (21.3, 19.7, 23.1))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "writegrid")),
                    reason="reference writegrid not built")
def test_writegrid_matches_reference_binary(tree):
    root, name, ads = tree
    r1 = _run(os.path.join(BIN, "writegrid"), str(root), name, ads)
    assert r1.returncode == 0, r1.stdout
    from emptyroom_b200 import files
    gpath = os.path.join(root, "data", "grids", f"{name}_{ads}_SYNFF.txt")
    ours = files.read_grid_txt(gpath)
    ours_out = read_out(os.path.join(root, "output_files", f"{name}_{ads}_grid.out"))
    r2 = _run(os.path.join(REF, "writegrid"), str(root), name, ads)
    assert r2.returncode == 0, r2.stdout
    theirs = files.read_grid_txt(gpath)
    theirs_out = read_out(os.path.join(root, "output_files", f"{name}_{ads}_grid.out"))
    assert ours.shape == theirs.shape
    s, P, rep = particles_from_tree(str(root), name, "SYNFF", ads)
    S = oracle.grid_abs(P, s.t_matrix, rep, 12.5 * 12.5, ours.shape)
    st = grid_errors(ours, theirs, S + 1e-6 * np.abs(theirs) / 2e-6)
    assert st["neg_ok"] and st["pos_ok"], st
    # reports: identical apart from the lines that describe each GPU layout
    impl = ("    Size of grid", "    A block is")
    a = [ln for ln in ours_out if not ln.startswith(impl)]
    b = [ln for ln in theirs_out if not ln.startswith(impl)]
    assert a == b


def test_writegrid_cube(tree):
    root, name, ads = tree
    sim = os.path.join(root, "simulation.input")
    txt = open(sim).read().replace("GridOutputFormat txt", "GridOutputFormat cube")
    open(sim, "w").write(txt)
    r = _run(os.path.join(BIN, "writegrid"), str(root), name, ads)
    assert r.returncode == 0, r.stdout
    lines = open(os.path.join(root, "data", "grids", f"{name}_{ads}_SYNFF.cube")).read().splitlines()
    assert lines[1] == "This is a grid file." and lines[3].split()[0] == str(int(np.ceil(21.3 / 0.7)))


def _kh(path):
    txt = open(path).read()
    m = re.search(r"Henry coefficient \(mol/\(m3-Pa\)\): (\S+)", txt)
    e = re.search(r"<energy> \(K\): (\S+)", txt)
    return float(m.group(1)), float(e.group(1))


def test_henry_tool_and_reference(tree):
    root, name, ads = tree
    r = _run(os.path.join(BIN, "henry"), str(root), name, ads)
    assert r.returncode == 0, r.stdout + r.stderr
    out = os.path.join(root, "output_files", f"{name}_{ads}_henry.out")
    kh, e_mean = _kh(out)
    assert kh > 0
    lines = read_out(out)
    assert "    # of blocks: 64" in lines and "Henry simulation results" in lines
    # same count as the reference's decomposition, same Philox points as the oracle
    n_line = [ln for ln in lines if ln.startswith("    Total # of insertions:")][0]
    n_tot = int(n_line.split(":")[1])
    assert n_tot % 16384 == 0
    s, P, rep = particles_from_tree(str(root), name, "SYNFF", ads)
    o = oracle.henry(P, s.t_matrix, rep, 12.5 * 12.5, 298.0, 1234, n_tot)
    kh_o = o["sum_w"] / n_tot / 298.0 / 8.314
    assert abs(kh - kh_o) <= 1e-5 * kh_o  # .out holds 7 significant digits
    if os.path.exists(os.path.join(REF, "henry")):
        r2 = _run(os.path.join(REF, "henry"), str(root), name, ads)
        assert r2.returncode == 0, r2.stdout
        kh_ref, _ = _kh(out)
        ref_lines = read_out(out)
        # identical reports up to the results (different random streams)
        cut = ref_lines.index("Henry simulation results")
        assert lines[:cut] == ref_lines[:cut]
        # statistical agreement of two independent estimates of K_H
        assert abs(kh - kh_ref) <= 0.05 * kh_ref
