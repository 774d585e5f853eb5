"""The benchmark's seeded frameworks, built with the oracle's generators only.

TEST INFRASTRUCTURE ONLY. The benchmark's reference arm times the reference's
CPU code on the same frameworks as the GPU arm without loading the library it
is compared with. These functions draw exactly what the GPU arm's workload
generator draws (same NumPy streams, same cell matrices, replication factors
and random sequential addition, restated in er_oracle_synth.c), so the two
arms see identical inputs; tests/test_oracle_pin.py checks that bit for bit.
Lorentz-Berthelot mixing follows src/load_fast_particle_f_array.h:35-36.
"""
from __future__ import annotations

import math

import numpy as np

from . import cell_matrices, replication_factors, synth_positions

PROBES = {  # label: (epsilon K, sigma A)
    "CH4": (148.0, 3.73),
    "Xe": (221.0, 4.10),
    "Kr": (166.4, 3.636),
}
MAX_DENSITY = 0.16  # atoms / A^3: the config-2 atom counts are capped here


class Framework:
    def __init__(self, name, t_matrix, frac, types, type_eps, type_sig, probe, rc, rep, dims):
        self.name = name
        self.t_matrix = t_matrix
        self.frac = frac
        self.types = types
        self.type_eps = type_eps
        self.type_sig = type_sig
        self.probe = probe
        self.rc = rc
        self.rep = rep
        self.dims = dims

    @property
    def rc2(self):
        return self.rc * self.rc

    def particles(self):
        """(N, 5) FrameworkParticle rows: x_f, y_f, z_f, eps_mix, sig_mix^2."""
        pe, ps = PROBES[self.probe]
        eps_f = self.type_eps[self.types]
        sig_f = self.type_sig[self.types]
        out = np.empty((len(self.frac), 5))
        out[:, :3] = self.frac
        out[:, 3] = np.sqrt(pe * eps_f)
        out[:, 4] = ((ps + sig_f) / 2.0) ** 2
        return out


def framework(seed, abc, angles, n_atoms, n_types, probe, rc, d_min, dims, name):
    rng = np.random.default_rng(seed)
    t, _, _ = cell_matrices(*abc, *angles)
    frac = synth_positions(seed, t, n_atoms, d_min)
    types = rng.integers(0, n_types, size=n_atoms)
    type_eps = rng.uniform(20.0, 100.0, size=n_types)
    type_sig = rng.uniform(2.5, 3.8, size=n_types)
    return Framework(name, t, frac, types, type_eps, type_sig, probe, rc,
                     replication_factors(t, rc), tuple(dims))


def grid_dims_for(abc, spacing):
    """N_i = ceil(L_i / resolution), src/writegrid.cu:110-112."""
    return tuple(int(math.ceil(L / spacing)) for L in abc)


def config2(n_frameworks=256, seed=1000, spacing_range=(0.1, 0.2)):
    """The 256 triclinic frameworks of the batch workload (a, b, c ~ U[8, 40] A,
    angles ~ U[60, 120] deg, 100-5000 atoms log-uniform capped at 0.16 / A^3,
    8 types, probes CH4 / Xe / Kr, spacing ~ U[0.1, 0.2] A)."""
    rng = np.random.default_rng(seed)
    out = []
    probes = list(PROBES)
    k = 0
    while len(out) < n_frameworks:
        abc = tuple(float(x) for x in rng.uniform(8.0, 40.0, size=3))
        ang = tuple(float(x) for x in rng.uniform(60.0, 120.0, size=3))
        try:
            _, _, vol = cell_matrices(*abc, *ang)
        except ValueError:
            continue
        n = int(round(math.exp(rng.uniform(math.log(100), math.log(5000)))))
        n = max(1, min(n, int(MAX_DENSITY * vol)))
        probe = probes[int(rng.integers(0, 3))]
        spacing = float(rng.uniform(*spacing_range))
        out.append(framework(seed + 1 + k, abc, ang, n, 8, probe, 12.5, 1.2,
                             grid_dims_for(abc, spacing), f"config2_{len(out)}"))
        k += 1
    return out


def config4(n_frameworks=64, seed=4000, spacing=0.2):
    """The Widom batch: config-1 cells (cubic 25.8 A, 424 atoms, 4 types), Xe."""
    abc = (25.8, 25.8, 25.8)
    dims = grid_dims_for(abc, spacing)
    return [framework(seed + k, abc, (90.0, 90.0, 90.0), 424, 4, "Xe", 12.5, 1.2, dims,
                      f"config4_{k}") for k in range(n_frameworks)]
