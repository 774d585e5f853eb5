"""Seeded synthetic frameworks for the benchmark workloads.

No public dataset ships with the reference, so every workload is generated:
cells, atom positions (random sequential addition with a minimum distance,
``er_synth_positions``), atom types with epsilon/sigma drawn uniformly, and
Lorentz-Berthelot mixing with the probe (src/load_fast_particle_f_array.h:35-36).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import cell_matrices, lorentz_berthelot, particles, replication_factors, synth_positions

PROBES = {  # label: (epsilon K, sigma A)
    "CH4": (148.0, 3.73),
    "Xe": (221.0, 4.10),
    "Kr": (166.4, 3.636),
}


@dataclass
class SynthFramework:
    name: str
    abc: tuple
    angles: tuple
    t_matrix: np.ndarray
    volume: float
    frac: np.ndarray          # (N, 3)
    types: np.ndarray         # (N,) int
    type_eps: np.ndarray      # (n_types,) K
    type_sig: np.ndarray      # (n_types,) A
    probe: str
    rc: float
    rep: tuple
    dims: tuple = (32, 32, 32)
    meta: dict = field(default_factory=dict)

    @property
    def n_atoms(self):
        return len(self.frac)

    def particles(self, probe=None):
        pe, ps = PROBES[probe or self.probe]
        eps, sig2 = lorentz_berthelot(self.type_eps[self.types], self.type_sig[self.types], pe, ps)
        return particles(self.frac, eps, sig2)

    @property
    def rc2(self):
        return self.rc * self.rc


def make_framework(seed, abc, angles, n_atoms, n_types=4, probe="CH4", rc=12.5, d_min=1.2,
                   dims=(32, 32, 32), name=None):
    rng = np.random.default_rng(seed)
    t, _, vol = cell_matrices(*abc, *angles)
    frac = synth_positions(seed, t, n_atoms, d_min)
    types = rng.integers(0, n_types, size=n_atoms)
    type_eps = rng.uniform(20.0, 100.0, size=n_types)
    type_sig = rng.uniform(2.5, 3.8, size=n_types)
    rep = replication_factors(t, rc)
    return SynthFramework(name or f"syn{seed}", tuple(abc), tuple(angles), t, vol, frac, types,
                          type_eps, type_sig, probe, rc, rep, tuple(dims))


def config1(seed=0):
    """Cubic 25.8 A, 424 atoms (d_min 1.2 A), 4 types, CH4, rc 12.5, 32^3 grid."""
    return make_framework(seed, (25.8, 25.8, 25.8), (90.0, 90.0, 90.0), 424, n_types=4,
                          probe="CH4", rc=12.5, d_min=1.2, dims=(32, 32, 32),
                          name=f"config1_s{seed}")


def grid_dims_for(abc, spacing):
    """N_i = ceil(L_i / resolution), src/writegrid.cu:110-112."""
    return tuple(int(math.ceil(L / spacing)) for L in abc)


# Number density above which the 1.2 A minimum distance of the config-1
# generator is no longer reachable by random sequential addition in
# reasonable time; config-2 atom counts are capped at this density.
MAX_DENSITY = 0.16


def config2(n_frameworks=256, seed=1000, spacing_range=(0.1, 0.2), max_density=MAX_DENSITY):
    """256 triclinic cells: a,b,c ~ U[8,40] A, angles ~ U[60,120] deg (valid cells),
    N log-uniform in [100, 5000] (capped at max_density * V), 8 types, probes
    CH4/Xe/Kr, grid spacing ~ U[0.1, 0.2] A."""
    rng = np.random.default_rng(seed)
    out = []
    probes = list(PROBES)
    k = 0
    while len(out) < n_frameworks:
        abc = tuple(float(x) for x in rng.uniform(8.0, 40.0, size=3))
        ang = tuple(float(x) for x in rng.uniform(60.0, 120.0, size=3))
        try:
            t, _, vol = cell_matrices(*abc, *ang)
        except Exception:
            continue
        n = int(round(math.exp(rng.uniform(math.log(100), math.log(5000)))))
        n_cap = int(max_density * vol)
        capped = n > n_cap
        n = max(1, min(n, n_cap))
        probe = probes[int(rng.integers(0, 3))]
        spacing = float(rng.uniform(*spacing_range))
        dims = grid_dims_for(abc, spacing)
        fw = make_framework(seed + 1 + k, abc, ang, n, n_types=8, probe=probe, rc=12.5,
                            d_min=1.2, dims=dims, name=f"config2_{len(out)}")
        fw.meta.update(spacing=spacing, n_drawn_capped=capped)
        out.append(fw)
        k += 1
    return out


def config3(seed=3):
    """One 4096-atom triclinic cell (30.1, 32.4, 28.7; 85/95/110 deg), CH4, 256^3."""
    return make_framework(seed, (30.1, 32.4, 28.7), (85.0, 95.0, 110.0), 4096, n_types=4,
                          probe="CH4", rc=12.5, d_min=1.2, dims=(256, 256, 256),
                          name="config3")


def config4(n_frameworks=64, seed=4000, spacing=0.2):
    """Widom batch: 64 config-1 cells (cubic 25.8 A, 424 atoms, d_min 1.2 A, 4
    types), Xe probe, pocket-blocking grid at 0.2 A (130^3)."""
    abc = (25.8, 25.8, 25.8)
    dims = grid_dims_for(abc, spacing)
    return [make_framework(seed + k, abc, (90.0, 90.0, 90.0), 424, n_types=4, probe="Xe",
                           rc=12.5, d_min=1.2, dims=dims, name=f"config4_{k}")
            for k in range(n_frameworks)]


def config5_stream(seed=5000, rate=200.0, seconds=60.0, n_frameworks=32, grid_fraction=0.7,
                   atoms=(50, 10000), insertions=(1_000_000, 10_000_000),
                   spacing_range=(0.1, 0.2), max_density=MAX_DENSITY):
    """Serving stream: Poisson arrivals at `rate` jobs/s for `seconds`; 70 %
    grid jobs (spacing ~ U[0.1, 0.2] A), 30 % Henry jobs (insertions
    log-uniform in [1e6, 1e7]); a pool of frameworks with the config-1 cell
    (cubic 25.8 A), 4 types, atom counts log-uniform in [50, 10000] capped at
    max_density * V, probes uniform over CH4 / Xe / Kr.
    Returns (frameworks, jobs); a job is a dict with t (arrival, s), kind
    ("grid" | "henry"), fw (pool index), dims or n_ins, seed."""
    rng = np.random.default_rng(seed)
    abc = (25.8, 25.8, 25.8)
    t_, _, vol = cell_matrices(*abc, 90.0, 90.0, 90.0)
    probes = list(PROBES)
    fws = []
    for k in range(n_frameworks):
        n = int(round(math.exp(rng.uniform(math.log(atoms[0]), math.log(atoms[1])))))
        n = max(1, min(n, int(max_density * vol)))
        fws.append(make_framework(seed + 1 + k, abc, (90.0, 90.0, 90.0), n, n_types=4,
                                  probe=probes[int(rng.integers(0, 3))], rc=12.5, d_min=1.2,
                                  name=f"config5_{k}"))
    jobs = []
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= seconds:
            break
        fw = int(rng.integers(0, n_frameworks))
        if rng.random() < grid_fraction:
            dims = grid_dims_for(abc, float(rng.uniform(*spacing_range)))
            jobs.append({"t": t, "kind": "grid", "fw": fw, "dims": dims})
        else:
            n_ins = int(round(math.exp(rng.uniform(math.log(insertions[0]),
                                                   math.log(insertions[1])))))
            jobs.append({"t": t, "kind": "henry", "fw": fw, "n_ins": n_ins,
                         "seed": int(rng.integers(0, 2**31))})
    return fws, jobs
