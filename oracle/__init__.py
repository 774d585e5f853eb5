"""CPU checkers for the CUDA path (test infrastructure only).

Two libraries, both loaded through ctypes:

* ``liboracle.so`` (``er_oracle.c``): this repository's FP64 restatement of
  the reference's grid / Widom / pocket-blocking algorithms.
* ``_ref/libref.so``: the reference's own code (``src/computegridsheet.h``,
  ``src/pocketblocking.cc``, ``src/Framework.cc``, ``src/Forcefield.cc``)
  compiled from its sources by ``oracle/Makefile``; optional.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs import this package. The product never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)

_lib = None
_ref = None


def _ptr(a, t):
    return a.ctypes.data_as(t)


def lib():
    """The restatement library (built by ``make -C oracle``)."""
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        L = ctypes.CDLL(path)
        L.oracle_point_energy.restype = ctypes.c_double
        L.oracle_point_energy.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double]
        L.oracle_grid.restype = None
        L.oracle_grid.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        L.oracle_points.restype = None
        L.oracle_points.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                    ctypes.c_double, _dp, ctypes.c_int64, _dp, ctypes.c_int]
        L.oracle_points_pairs.restype = None
        L.oracle_points_pairs.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                          ctypes.c_double, _dp, ctypes.c_int64, _dp,
                                          ctypes.c_int]
        L.oracle_points_abs.restype = None
        L.oracle_points_abs.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                        ctypes.c_double, _dp, ctypes.c_int64, _dp, ctypes.c_int]
        L.oracle_accessibility.restype = None
        L.oracle_accessibility.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _u8p, ctypes.c_int]
        L.oracle_philox4x32_10.restype = None
        L.oracle_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.oracle_insertion_points.restype = None
        L.oracle_insertion_points.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64,
                                              _dp]
        L.oracle_insertion_point.restype = None
        L.oracle_insertion_point.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _dp]
        L.oracle_henry.restype = None
        L.oracle_henry.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_uint64, ctypes.c_int64, _u8p,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                   ctypes.c_int]
        L.oracle_block_pockets.restype = ctypes.c_int
        L.oracle_block_pockets.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, _ip]
        L.oracle_grid_interp.restype = None
        L.oracle_grid_interp.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                         ctypes.c_int64, _dp]
        L.oracle_points_cells.restype = ctypes.c_int
        L.oracle_points_cells.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                          ctypes.c_double, _dp, ctypes.c_int64, _dp, _dp, _dp,
                                          ctypes.c_int]
        L.oracle_grid_cells.restype = ctypes.c_int
        L.oracle_grid_cells.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                        ctypes.c_int]
        L.oracle_henry_cells.restype = ctypes.c_int
        L.oracle_henry_cells.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_uint64, ctypes.c_int64, _u8p,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                         ctypes.c_int]
        L.oracle_cell_matrices.restype = ctypes.c_int
        L.oracle_cell_matrices.argtypes = [ctypes.c_double] * 6 + [_dp, _dp, _dp]
        L.oracle_replication_factors.restype = ctypes.c_int
        L.oracle_replication_factors.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _ip]
        L.oracle_synth_positions.restype = ctypes.c_int
        L.oracle_synth_positions.argtypes = [ctypes.c_uint64, _dp, ctypes.c_int, ctypes.c_double,
                                             _dp]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref.so"))


def ref():
    """The reference's own code compiled as host C++ (None when not built)."""
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libref.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_grid.restype = None
        R.ref_grid.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double, ctypes.c_int,
                               ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        R.ref_grid_sheets.restype = None
        R.ref_grid_sheets.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, ctypes.c_int,
                                      _dp, ctypes.c_int]
        R.ref_points.restype = None
        R.ref_points.argtypes = [_dp, ctypes.c_int, _dp, _ip, ctypes.c_double, _dp,
                                 ctypes.c_int64, _dp, ctypes.c_int]
        R.ref_accessibility.restype = None
        R.ref_accessibility.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _dp, ctypes.c_int]
        R.ref_block_pockets.restype = ctypes.c_int
        R.ref_block_pockets.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double]
        R.ref_load_framework.restype = ctypes.c_int
        R.ref_load_framework.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _dp, _dp,
                                         ctypes.c_int]
        if hasattr(R, "ref_grid_interp"):
            R.ref_grid_interp.restype = None
            R.ref_grid_interp.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                          ctypes.c_int64, _dp]
        R.ref_load_forcefield.restype = ctypes.c_int
        R.ref_load_forcefield.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _dp, _dp,
                                          ctypes.c_int]
        _ref = R
    return _ref


def _prep(particles, t, rep):
    p = np.ascontiguousarray(particles, dtype=np.float64).reshape(-1, 5)
    tm = np.ascontiguousarray(t, dtype=np.float64).reshape(9)
    r = np.ascontiguousarray(rep, dtype=np.int32).reshape(3)
    return p, tm, r


# --------------------------------------------------------------- restatement
def grid(particles, t, rep, rc2, dims, n_threads=0):
    """FP64 grid, shape (nx, ny, nz), axes i/(N-1)."""
    p, tm, r = _prep(particles, t, rep)
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, dtype=np.float64)
    lib().oracle_grid(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2), nx, ny, nz,
                      _ptr(out, _dp), int(n_threads))
    return out.reshape(nx, ny, nz)


def points(particles, t, rep, rc2, pts, min_r=1e-12, n_threads=0):
    p, tm, r = _prep(particles, t, rep)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(q), dtype=np.float64)
    lib().oracle_points(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2),
                        float(min_r), _ptr(q, _dp), len(q), _ptr(out, _dp), int(n_threads))
    return out


def points_pairs(particles, t, rep, rc2, pts, min_r=1e-12, n_threads=0):
    """In-cutoff pair-term count at each point (float64 counts)."""
    p, tm, r = _prep(particles, t, rep)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(q), dtype=np.float64)
    lib().oracle_points_pairs(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2),
                              float(min_r), _ptr(q, _dp), len(q), _ptr(out, _dp),
                              int(n_threads))
    return out


def points_abs(particles, t, rep, rc2, pts, min_r=1e-12, n_threads=0):
    """Sum of |term| over the in-cutoff terms at each point (FP32 error scale)."""
    p, tm, r = _prep(particles, t, rep)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(q), dtype=np.float64)
    lib().oracle_points_abs(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2),
                            float(min_r), _ptr(q, _dp), len(q), _ptr(out, _dp), int(n_threads))
    return out


def lattice_points(dims):
    """Fractional coordinates i/(N-1) of every grid point, grid order."""
    nx, ny, nz = (int(d) for d in dims)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    return np.stack([ii / (nx - 1), jj / (ny - 1), kk / (nz - 1)], axis=-1).reshape(-1, 3)


def grid_abs(particles, t, rep, rc2, dims, n_threads=0):
    return points_abs(particles, t, rep, rc2, lattice_points(dims), 1e-12,
                      n_threads).reshape(tuple(int(d) for d in dims))


def accessibility(particles, t, dims, n_threads=0):
    p, tm, _ = _prep(particles, t, (1, 1, 1))
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, dtype=np.uint8)
    lib().oracle_accessibility(_ptr(p, _dp), len(p), _ptr(tm, _dp), nx, ny, nz,
                               _ptr(out, _u8p), int(n_threads))
    return out.reshape(nx, ny, nz)


def philox4x32_10(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(4)
    k = np.ascontiguousarray(key, dtype=np.uint32).reshape(2)
    o = np.empty(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_ptr(c, _u32p), _ptr(k, _u32p), _ptr(o, _u32p))
    return o


def insertion_point(seed, i):
    o = np.empty(3, dtype=np.float64)
    lib().oracle_insertion_point(int(seed), int(i), _ptr(o, _dp))
    return o


def insertion_points(seed, n, i0=0):
    """Insertion points i0 .. i0 + n - 1 of Philox stream `seed` (n x 3)."""
    o = np.empty((int(n), 3), dtype=np.float64)
    lib().oracle_insertion_points(int(seed), int(i0), int(n), _ptr(o, _dp))
    return o


def henry(particles, t, rep, rc2, T, seed, n_ins, mask=None, want_energies=False,
          n_threads=0):
    """Returns dict(sum_w, sum_ew, n, max_neg_e_over_t, n_blocked[, energies])."""
    p, tm, r = _prep(particles, t, rep)
    out = np.zeros(5, dtype=np.float64)
    en = np.empty(int(n_ins), dtype=np.float64) if want_energies else None
    if mask is not None:
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        mnx, mny, mnz = m.shape
        mp = _ptr(m, _u8p)
    else:
        mnx = mny = mnz = 0
        mp = None
    lib().oracle_henry(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2), float(T),
                       int(seed), int(n_ins), mp, mnx, mny, mnz, _ptr(out, _dp),
                       _ptr(en, _dp) if en is not None else None, int(n_threads))
    res = dict(sum_w=out[0], sum_ew=out[1], n=out[2], max_neg_e_over_t=out[3],
               n_blocked=int(out[4]))
    if en is not None:
        res["energies"] = en
    return res


# ------------------------------------------------ cell-list form of the sums
def points_cells(particles, t, rep, rc2, pts, min_r=1e-12, n_threads=0):
    """(energy, sum |term|, in-cutoff count) per point: the terms of `points`
    summed cell by cell (er_oracle_cells.c)."""
    p, tm, r = _prep(particles, t, rep)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    e = np.empty(len(q)); s = np.empty(len(q)); c = np.empty(len(q))
    st = lib().oracle_points_cells(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip),
                                   float(rc2), float(min_r), _ptr(q, _dp), len(q), _ptr(e, _dp),
                                   _ptr(s, _dp), _ptr(c, _dp), int(n_threads))
    if st:
        raise MemoryError("oracle_points_cells")
    return e, s, c


def grid_cells(particles, t, rep, rc2, dims, n_threads=0, want_abs=False):
    """FP64 grid (and sum |term| per point) by the cell-list sum."""
    p, tm, r = _prep(particles, t, rep)
    nx, ny, nz = (int(d) for d in dims)
    e = np.empty(nx * ny * nz)
    s = np.empty(nx * ny * nz) if want_abs else None
    st = lib().oracle_grid_cells(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2),
                                 nx, ny, nz, _ptr(e, _dp), _ptr(s, _dp) if want_abs else None,
                                 int(n_threads))
    if st:
        raise MemoryError("oracle_grid_cells")
    e = e.reshape(nx, ny, nz)
    return (e, s.reshape(nx, ny, nz)) if want_abs else e


def henry_cells(particles, t, rep, rc2, T, seed, n_ins, mask=None, want_energies=False,
                n_threads=0):
    """`henry` with the cell-list energies; same result keys."""
    p, tm, r = _prep(particles, t, rep)
    out = np.zeros(5, dtype=np.float64)
    en = np.empty(int(n_ins), dtype=np.float64) if want_energies else None
    if mask is not None:
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        mnx, mny, mnz = m.shape
        mp = _ptr(m, _u8p)
    else:
        mnx = mny = mnz = 0
        mp = None
    st = lib().oracle_henry_cells(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2),
                                  float(T), int(seed), int(n_ins), mp, mnx, mny, mnz,
                                  _ptr(out, _dp), _ptr(en, _dp) if en is not None else None,
                                  int(n_threads))
    if st:
        raise MemoryError("oracle_henry_cells")
    res = dict(sum_w=out[0], sum_ew=out[1], n=out[2], max_neg_e_over_t=out[3],
               n_blocked=int(out[4]))
    if en is not None:
        res["energies"] = en
    return res


# --------------------------------------------- generators of the workloads
def cell_matrices(a, b, c, alpha, beta, gamma):
    """(t_matrix 3x3, inv 3x3, volume), src/Framework.cc:113-142."""
    t = np.zeros(9); inv = np.zeros(9); v = np.zeros(1)
    if lib().oracle_cell_matrices(a, b, c, alpha, beta, gamma, _ptr(t, _dp), _ptr(inv, _dp),
                                  _ptr(v, _dp)):
        raise ValueError("degenerate cell")
    return t.reshape(3, 3), inv.reshape(3, 3), float(v[0])


def replication_factors(t, r_cutoff, factor=1):
    tm = np.ascontiguousarray(t, dtype=np.float64).reshape(9)
    rep = np.zeros(3, dtype=np.int32)
    if lib().oracle_replication_factors(_ptr(tm, _dp), float(r_cutoff), int(factor),
                                        _ptr(rep, _ip)):
        raise ValueError("replication factors")
    return tuple(int(x) for x in rep)


def synth_positions(seed, t, n_atoms, d_min):
    tm = np.ascontiguousarray(t, dtype=np.float64).reshape(9)
    out = np.empty((int(n_atoms), 3))
    if lib().oracle_synth_positions(int(seed), _ptr(tm, _dp), int(n_atoms), float(d_min),
                                    _ptr(out, _dp)):
        raise ValueError(f"could not place {n_atoms} atoms at d_min={d_min}")
    return out


def block_pockets(grid3, T):
    """Returns (blocked copy of the grid, n_pockets, segment ids)."""
    g = np.array(grid3, dtype=np.float64, copy=True, order="C")
    nx, ny, nz = g.shape
    seg = np.empty(g.size, dtype=np.int32)
    n = lib().oracle_block_pockets(_ptr(g, _dp), nx, ny, nz, float(T), _ptr(seg, _ip))
    return g, int(n), seg.reshape(g.shape)


# ------------------------------------------------------------ reference code
def ref_grid(particles, t, rep, rc2, dims, n_threads=0):
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    p, tm, r = _prep(particles, t, rep)
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, dtype=np.float64)
    R.ref_grid(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2), nx, ny, nz,
               _ptr(out, _dp), int(n_threads))
    return out.reshape(nx, ny, nz)


def ref_grid_sheets(particles, t, rep, rc2, dims, sheets, n_threads=0):
    """The reference's ComputeGridSheet for the listed x-sheets only (threads over
    sheets); returns an array (len(sheets), ny, nz). Used to time the reference
    on a bounded sample of a grid."""
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    p, tm, r = _prep(particles, t, rep)
    nx, ny, nz = (int(d) for d in dims)
    sh = np.ascontiguousarray(sheets, dtype=np.int32)
    out = np.empty(len(sh) * ny * nz, dtype=np.float64)
    R.ref_grid_sheets(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2), nx, ny,
                      nz, _ptr(sh, _ip), len(sh), _ptr(out, _dp), int(n_threads))
    return out.reshape(len(sh), ny, nz)


def ref_points(particles, t, rep, rc2, pts, n_threads=0):
    """The reference's ComputeGridSheet at arbitrary fractional points (n x 3)."""
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    p, tm, r = _prep(particles, t, rep)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(q), dtype=np.float64)
    R.ref_points(_ptr(p, _dp), len(p), _ptr(tm, _dp), _ptr(r, _ip), float(rc2), _ptr(q, _dp),
                 len(q), _ptr(out, _dp), int(n_threads))
    return out


def ref_accessibility(particles, t, dims, n_threads=0):
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    p, tm, _ = _prep(particles, t, (1, 1, 1))
    nx, ny, nz = (int(d) for d in dims)
    out = np.empty(nx * ny * nz, dtype=np.float64)
    R.ref_accessibility(_ptr(p, _dp), len(p), _ptr(tm, _dp), nx, ny, nz, _ptr(out, _dp),
                        int(n_threads))
    return out.reshape(nx, ny, nz).astype(np.uint8)


def ref_block_pockets(grid3, T):
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    g = np.array(grid3, dtype=np.float64, copy=True, order="C")
    nx, ny, nz = g.shape
    n = R.ref_block_pockets(_ptr(g, _dp), nx, ny, nz, float(T))
    return g, int(n)


def ref_load_framework(root, name, max_atoms=100000):
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    out = np.zeros(26, dtype=np.float64)
    frac = np.zeros(3 * max_atoms, dtype=np.float64)
    n = R.ref_load_framework(str(root).encode(), name.encode(), _ptr(out, _dp),
                             _ptr(frac, _dp), max_atoms)
    return dict(a=out[0], b=out[1], c=out[2], alpha=out[3], beta=out[4], gamma=out[5],
                volume=out[6], density=out[7], t_matrix=out[8:17].reshape(3, 3).copy(),
                inv_t_matrix=out[17:26].reshape(3, 3).copy(),
                frac=frac[:3 * n].reshape(n, 3).copy(), n_atoms=n)


def ref_load_forcefield(root, name, max_entries=10000):
    R = ref()
    if R is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    eps = np.zeros(max_entries)
    sig = np.zeros(max_entries)
    n = R.ref_load_forcefield(str(root).encode(), name.encode(), _ptr(eps, _dp),
                              _ptr(sig, _dp), max_entries)
    return eps[:n].copy(), sig[:n].copy()


def grid_interp(grid, pts):
    """GCMC trilinear lookup (src/gcmc.cc:145-177 at WrapToInterval(., 1)),
    restated; grid (nx, ny, nz) float64, pts (n, 3) fractional."""
    g = np.ascontiguousarray(grid, dtype=np.float64)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(q), dtype=np.float64)
    nx, ny, nz = g.shape
    lib().oracle_grid_interp(_ptr(g, _dp), nx, ny, nz, _ptr(q, _dp), len(q), _ptr(out, _dp))
    return out


def ref_grid_interp(grid, pts):
    """The reference's own GuestFrameworkEnergy / WrapToInterval (extracted from
    src/gcmc.cc at build time) on the same inputs."""
    R = ref()
    if R is None or not hasattr(R, "ref_grid_interp"):
        raise RuntimeError("oracle/_ref/libref.so not built with the GCMC lookup")
    g = np.array(grid, dtype=np.float64, order="C", copy=True)
    q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.empty(len(q), dtype=np.float64)
    nx, ny, nz = g.shape
    R.ref_grid_interp(_ptr(g, _dp), nx, ny, nz, _ptr(q, _dp), len(q), _ptr(out, _dp))
    return out
