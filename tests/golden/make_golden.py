"""Generates the golden fixtures in this folder from the reference's own code.

Run in a container where the reference tree exists (oracle/_ref/libref.so is
built from it by `make -C oracle`):

    python tests/golden/make_golden.py

Each fixture stores seeded inputs and the outputs that the reference's code
(src/computegridsheet.h kernels compiled as host C++, src/pocketblocking.cc,
src/Framework.cc, src/Forcefield.cc, the grid lookup of src/gcmc.cc) produced
for them, so tests can pin the
oracle restatement and the CUDA path on machines without the reference.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

import oracle  # noqa: E402
from emptyroom_b200 import synth  # noqa: E402


def grid_case(fw, dims):
    P = fw.particles()
    g = oracle.ref_grid(P, fw.t_matrix, fw.rep, fw.rc2, dims)
    acc = oracle.ref_accessibility(P, fw.t_matrix, dims)
    return dict(particles=P, t_matrix=fw.t_matrix, rep=np.array(fw.rep, dtype=np.int32),
                rc2=np.float64(fw.rc2), dims=np.array(dims, dtype=np.int32), grid=g,
                accessibility=acc)


def pocket_grid(seed, dims, T):
    """An energy field with pores, channels and pockets: blocked (E >= 15 T)
    wherever a smooth random field exceeds a level, plus a straight channel
    along x and a closed spherical pocket."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    x, y, z = np.meshgrid(np.linspace(0, 1, nx), np.linspace(0, 1, ny), np.linspace(0, 1, nz),
                          indexing="ij")
    f = np.zeros(dims)
    for _ in range(6):
        k = rng.integers(1, 4, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        f += np.cos(2 * np.pi * k[0] * x + ph[0]) * np.cos(2 * np.pi * k[1] * y + ph[1]) * \
            np.cos(2 * np.pi * k[2] * z + ph[2])
    E = np.where(f > 0.3, 20.0 * T, -10.0 * T) + rng.uniform(-T, T, size=dims)
    # a closed pocket: sphere of accessible points inside a blocked shell
    c = np.array([0.5, 0.5, 0.5])
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    E[(r > 0.12) & (r < 0.2)] = 30.0 * T
    E[r <= 0.12] = -5.0 * T
    # a periodic channel along x
    ch = (np.abs(y - 0.15) < 0.06) & (np.abs(z - 0.8) < 0.06)
    E[ch] = -8.0 * T
    return E


def percolation_grid(seed, dims, T, p_open):
    """Uncorrelated sites, open with probability p_open: near the percolation
    threshold this gives many segments, face-crossing pockets and channels."""
    rng = np.random.default_rng(seed)
    open_ = rng.random(dims) < p_open
    return np.where(open_, rng.uniform(-20 * T, 14.9 * T, size=dims),
                    rng.uniform(15 * T, 40 * T, size=dims))


def write_fixture_tree(root):
    """A tiny data/ tree in the reference's file formats (for the loaders)."""
    os.makedirs(os.path.join(root, "data", "structures"), exist_ok=True)
    os.makedirs(os.path.join(root, "data", "forcefields"), exist_ok=True)
    with open(os.path.join(root, "data", "structures", "SYN1.cssr"), "w") as fh:
        fh.write("\t\t\t\t21.100  23.300  19.700\n")
        fh.write("\t\t80  100  115  SPGR =  1 P 1\t\t OPT = 1\n")
        fh.write("6  0\n")
        fh.write("0 SYN1\t: SYN1\n")
        rows = [("Zn", 0.1, 0.2, 0.3), ("O", 0.5, 0.25, 0.75), ("C", 1.25, -0.5, 0.5),
                ("H", 0.99, 0.01, 0.5), ("C", 0.33, 0.66, 0.125), ("O", -0.25, 0.4, 1.0)]
        for i, (lab, a, b, c) in enumerate(rows):
            fh.write(f" {i + 1} {lab} {a:.6f} {b:.6f} {c:.6f}  0  0  0  0  0  0  0  0  0.000000\n")
    with open(os.path.join(root, "data", "masses.def"), "w") as fh:
        fh.write("[atom] [mass]\nZn 65.38\nO 15.999\nC 12.011\nH 1.008\nCH4 16.04\n")
    with open(os.path.join(root, "data", "forcefields", "SYNFF.def"), "w") as fh:
        fh.write("[Atom] [epsilon (K)] [sigma (A)]\nZn 62.4 2.46\nO 30.19 3.12\nC 52.83 3.43\n"
                 "H 22.14 2.57\nCH4 148.0 3.73\nXe 221.0 4.10\n")


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libref.so is not built; run make -C oracle first")
    out = {}
    fw1 = synth.config1(seed=11)
    out["grid_cubic"] = grid_case(fw1, (9, 10, 11))
    fwt = synth.make_framework(12, (14.2, 16.8, 13.1), (75.0, 104.0, 112.0), 50, n_types=4,
                               probe="Xe", rc=12.5, d_min=1.2, name="tri")
    out["grid_triclinic"] = grid_case(fwt, (8, 9, 7))
    fws = synth.make_framework(13, (9.0, 10.5, 8.5), (90.0, 90.0, 90.0), 14, n_types=3,
                               probe="Kr", rc=9.0, d_min=1.2, name="small")
    out["grid_rep2"] = grid_case(fws, (6, 6, 6))
    for key, (seed, dims, T) in {"pockets_a": (21, (20, 22, 18), 298.0),
                                 "pockets_b": (22, (15, 15, 15), 150.0)}.items():
        E = pocket_grid(seed, dims, T)
        blocked, n = oracle.ref_block_pockets(E, T)
        out[key] = dict(grid=E, T=np.float64(T), blocked=blocked, n_pockets=np.int32(n))
    for key, (seed, dims, T, p) in {"pockets_perc": (23, (16, 17, 15), 298.0, 0.30),
                                    "pockets_perc_dense": (24, (12, 12, 12), 77.0, 0.45),
                                    "pockets_sparse": (25, (14, 13, 12), 300.0, 0.18)}.items():
        E = percolation_grid(seed, dims, T, p)
        blocked, n = oracle.ref_block_pockets(E, T)
        out[key] = dict(grid=E, T=np.float64(T), blocked=blocked, n_pockets=np.int32(n))
    # GCMC lookup: a config-1 grid with two blocked pockets, points inside and
    # outside [0, 1) (the call sites wrap them)
    g1 = out["grid_cubic"]["grid"].copy()
    g1[2, 3, 4] = 1e13
    g1[6, 7, 8] = 1e13
    rng = np.random.default_rng(26)
    pts = np.concatenate([rng.uniform(0.0, 1.0, size=(400, 3)),
                          rng.uniform(-2.0, 3.0, size=(200, 3)),
                          np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5], [0.125, 0.25, 0.375]])])
    out["gcmc_interp"] = dict(grid=g1, pts=pts, energy=oracle.ref_grid_interp(g1, pts))
    # loaders on a fixture tree written in the reference's formats
    with tempfile.TemporaryDirectory() as tmp:
        write_fixture_tree(tmp)
        f = oracle.ref_load_framework(tmp, "SYN1")
        eps, sig = oracle.ref_load_forcefield(tmp, "SYNFF")
    out["loader_syn1"] = dict(a=f["a"], b=f["b"], c=f["c"], alpha=f["alpha"], beta=f["beta"],
                              gamma=f["gamma"], volume=f["volume"], density=f["density"],
                              t_matrix=f["t_matrix"], inv_t_matrix=f["inv_t_matrix"],
                              frac=f["frac"], ff_eps=eps, ff_sig=sig)
    for name, d in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                            **{k: np.asarray(v) for k, v in d.items()})
        print("wrote", name)


if __name__ == "__main__":
    main()
