"""The reference's file formats through the C ABI (er_structure_*, er_forcefield_*,
er_read_settings, er_write_grid_*): loaders for .cssr / .def / masses.def / .uc /
simulation.input and the grid text writers and reader."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import ErSettings

ER_SETTINGS_GRID = 1
ER_SETTINGS_HENRY = 2


class FileError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _err():
    return ctypes.create_string_buffer(1024)


def _b(s):
    return s.encode() if isinstance(s, str) else s


class Structure:
    """Framework(name): a .cssr file plus masses (src/Framework.cc)."""

    def __init__(self, root, name):
        h = ctypes.c_void_p()
        e = _err()
        st = _capi.lib().er_structure_load(_b(str(root)), _b(name), ctypes.byref(h), e, 1024)
        if st != 0:
            raise FileError(st, e.value.decode())
        self._h = h
        n = ctypes.c_int(0)
        cell = np.zeros(6)
        t = np.zeros(9)
        inv = np.zeros(9)
        vol = ctypes.c_double(0)
        dens = ctypes.c_double(0)
        dp = ctypes.POINTER(ctypes.c_double)
        _capi.lib().er_structure_info(h, ctypes.byref(n), cell.ctypes.data_as(dp),
                                      t.ctypes.data_as(dp), inv.ctypes.data_as(dp),
                                      ctypes.byref(vol), ctypes.byref(dens))
        self.n_atoms = n.value
        self.a, self.b, self.c, self.alpha, self.beta, self.gamma = cell
        self.t_matrix = t.reshape(3, 3)
        self.inv_t_matrix = inv.reshape(3, 3)
        self.volume = vol.value
        self.density = dens.value
        self.frac = np.zeros((self.n_atoms, 3))
        _capi.lib().er_structure_frac(h, self.frac.ctypes.data_as(dp))
        buf = ctypes.create_string_buffer(256)
        self.labels = []
        for i in range(self.n_atoms):
            _capi.lib().er_structure_label(h, i, buf, 256)
            self.labels.append(buf.value.decode())

    def close(self):
        if self._h:
            _capi.lib().er_structure_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Forcefield:
    """Forcefield(name): a .def file (src/Forcefield.cc)."""

    def __init__(self, root, name):
        h = ctypes.c_void_p()
        e = _err()
        st = _capi.lib().er_forcefield_load(_b(str(root)), _b(name), ctypes.byref(h), e, 1024)
        if st != 0:
            raise FileError(st, e.value.decode())
        self._h = h
        n = _capi.lib().er_forcefield_count(h)
        self.labels, self.eps, self.sig = [], [], []
        buf = ctypes.create_string_buffer(256)
        for i in range(n):
            ep = ctypes.c_double(0)
            sg = ctypes.c_double(0)
            _capi.lib().er_forcefield_entry(h, i, buf, 256, ctypes.byref(ep), ctypes.byref(sg))
            self.labels.append(buf.value.decode())
            self.eps.append(ep.value)
            self.sig.append(sg.value)

    def find(self, label):
        ep = ctypes.c_double(0)
        sg = ctypes.c_double(0)
        st = _capi.lib().er_forcefield_find(self._h, _b(label), ctypes.byref(ep), ctypes.byref(sg))
        if st != 0:
            raise FileError(st, f"{label} not in force field")
        return ep.value, sg.value

    def close(self):
        if self._h:
            _capi.lib().er_forcefield_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mix_particles(structure, forcefield, eps_guest, sig_guest):
    out = np.zeros((structure.n_atoms, 5))
    e = _err()
    st = _capi.lib().er_mix_particles(structure._h, forcefield._h, float(eps_guest),
                                      float(sig_guest), out.ctypes.data_as(ctypes.c_void_p), e,
                                      1024)
    if st != 0:
        raise FileError(st, e.value.decode())
    return out


def adsorbate_mw(root, adsorbate):
    v = ctypes.c_double(0)
    e = _err()
    st = _capi.lib().er_adsorbate_mw(_b(str(root)), _b(adsorbate), ctypes.byref(v), e, 1024)
    if st != 0:
        raise FileError(st, e.value.decode())
    return v.value


def read_uc(root, name, which="once"):
    rep = (ctypes.c_int * 3)()
    e = _err()
    st = _capi.lib().er_read_uc(_b(str(root)), _b(name), _b(which), rep, e, 1024)
    if st != 0:
        raise FileError(st, e.value.decode())
    return tuple(rep)


def write_uc(root, name, which, rep):
    r = (ctypes.c_int * 3)(*[int(x) for x in rep])
    st = _capi.lib().er_write_uc(_b(str(root)), _b(name), _b(which), r)
    if st != 0:
        raise FileError(st, "could not write .uc file")


def read_settings(path, kind):
    s = ErSettings()
    e = _err()
    st = _capi.lib().er_read_settings(_b(str(path)), int(kind), ctypes.byref(s), e, 1024)
    if st != 0:
        raise FileError(st, e.value.decode())
    return {"forcefield": s.forcefield.decode(), "verbose": s.verbose,
            "grid_resolution": s.grid_resolution,
            "grid_output_format": s.grid_output_format.decode(),
            "r_cutoff_squared": s.r_cutoff_squared, "feynman_hibbs": s.feynman_hibbs,
            "energy_threshold": s.energy_threshold, "temperature": s.temperature,
            "insertions_per_a3": s.insertions_per_a3}


def write_grid_txt(path, grid, n_threads=0):
    g = np.ascontiguousarray(grid, dtype=np.float32)
    nx, ny, nz = g.shape
    st = _capi.lib().er_write_grid_txt(_b(str(path)),
                                       g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       nx, ny, nz, int(n_threads))
    if st != 0:
        raise FileError(st, f"could not write {path}")


def write_grid_cube(path, grid, t_matrix, n_threads=0):
    g = np.ascontiguousarray(grid, dtype=np.float32)
    t = np.ascontiguousarray(t_matrix, dtype=np.float64).reshape(9)
    nx, ny, nz = g.shape
    st = _capi.lib().er_write_grid_cube(_b(str(path)),
                                        g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nx, ny,
                                        nz, t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        int(n_threads))
    if st != 0:
        raise FileError(st, f"could not write {path}")


def read_grid_txt(path):
    dims = (ctypes.c_int * 3)()
    e = _err()
    st = _capi.lib().er_read_grid_txt(_b(str(path)), None, 0, dims, e, 1024)
    if st != 0:
        raise FileError(st, e.value.decode())
    out = np.empty(tuple(dims), dtype=np.float64)
    st = _capi.lib().er_read_grid_txt(_b(str(path)),
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      out.size, dims, e, 1024)
    if st != 0:
        raise FileError(st, e.value.decode())
    return out
