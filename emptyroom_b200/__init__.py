"""emptyroom_b200 -- B200 (sm_100a) adsorption hot path of CorySimon/EmptyRoom.

The compute lives in ``libemptyroom_b200.so`` (hand-written CUDA kernels behind
the C ABI of ``include/emptyroom_b200.h``). This module is a thin host-side
mirror of that ABI for Python callers (tests, benchmarks, notebooks); the
drop-in command-line tools ``writegrid`` and ``henry`` are C++
(``emptyroom_b200/cli``). There is no CPU fallback: every compute call goes
through the library and fails loudly when it is missing or has no GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import ErFrameworkDesc, ErGridJob, ErHenryResult, ErParticle

ER_OK = 0
ER_OUT_HOST = 0x0
ER_OUT_DEVICE = 0x1
ER_OUT_F32 = 0x0
ER_OUT_F64 = 0x2
ER_PREC_NEAR64 = 0x0  # default: near pairs in FP64
ER_PREC_COMP = 0x08
ER_PREC_FP32 = 0x10
ER_PREC_FP64 = 0x20
ER_COUNT_PAIRS = 0x40
ER_TILE_P8 = 0x80
ER_BATCH_PERSISTENT = 0
ER_BATCH_PLAIN = 1
ER_BATCH_HOST_OUT = 0x100
ER_BATCH_AUTOTUNE = 0x200
ER_BATCH_COMP = 0x400
ER_ENERGY_CAP = 1.0e30
ER_INTERP_GRID_F64 = 0x1
R_GAS = 8.314  # J/(mol K), src/henry.cu:169


class ErError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _dptr(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def lorentz_berthelot(eps_f, sig_f, eps_g, sig_g):
    """Mixed (eps, sigma^2), src/load_fast_particle_f_array.h:35-36."""
    eps_f = np.asarray(eps_f, dtype=np.float64)
    sig_f = np.asarray(sig_f, dtype=np.float64)
    return np.sqrt(eps_g * eps_f), ((sig_g + sig_f) / 2.0) ** 2


def particles(frac, eps_mix, sig2_mix):
    """(N, 5) float64 array in FrameworkParticle order."""
    frac = np.asarray(frac, dtype=np.float64).reshape(-1, 3)
    out = np.empty((len(frac), 5), dtype=np.float64)
    out[:, :3] = frac
    out[:, 3] = eps_mix
    out[:, 4] = sig2_mix
    return out


def cell_matrices(a, b, c, alpha, beta, gamma):
    """(t_matrix, inv_t_matrix, volume) from lengths (A) and angles (deg)."""
    t = np.zeros(9)
    inv = np.zeros(9)
    v = ctypes.c_double(0.0)
    st = _capi.lib().er_cell_matrices(a, b, c, alpha, beta, gamma, _dptr(t), _dptr(inv),
                                      ctypes.byref(v))
    if st != ER_OK:
        raise ErError(st, "degenerate cell")
    return t.reshape(3, 3), inv.reshape(3, 3), v.value


def replication_factors(t_matrix, r_cutoff, factor=1):
    t = np.ascontiguousarray(t_matrix, dtype=np.float64).reshape(9)
    rep = np.zeros(3, dtype=np.int32)
    st = _capi.lib().er_replication_factors(_dptr(t), r_cutoff, factor,
                                            rep.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if st != ER_OK:
        raise ErError(st, "replication factors")
    return tuple(int(x) for x in rep)


def philox4x32_10(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(4)
    k = np.ascontiguousarray(key, dtype=np.uint32).reshape(2)
    o = np.empty(4, dtype=np.uint32)
    _capi.lib().er_philox4x32_10(_dptr(c, ctypes.c_uint32), _dptr(k, ctypes.c_uint32),
                                 _dptr(o, ctypes.c_uint32))
    return o


def insertion_point(seed, i):
    o = np.empty(3)
    _capi.lib().er_insertion_point(int(seed), int(i), _dptr(o))
    return o


def synth_positions(seed, t_matrix, n_atoms, d_min):
    t = np.ascontiguousarray(t_matrix, dtype=np.float64).reshape(9)
    out = np.empty((int(n_atoms), 3))
    st = _capi.lib().er_synth_positions(int(seed), _dptr(t), int(n_atoms), float(d_min),
                                        _dptr(out))
    if st != ER_OK:
        raise ErError(st, f"could not place {n_atoms} atoms at d_min={d_min}")
    return out


def version():
    return _capi.lib().er_version().decode()


class Framework:
    """A framework/probe pair resident on the device."""

    def __init__(self, ctx, fw_id, n_atoms):
        self.ctx = ctx
        self.id = fw_id
        self.n_atoms = n_atoms

    def release(self):
        if self.id is not None and self.ctx._h:
            self.ctx._check(_capi.lib().er_framework_release(self.ctx._h, self.id))
        self.id = None

    @property
    def device_bytes(self):
        n = ctypes.c_size_t(0)
        self.ctx._check(_capi.lib().er_framework_bytes(self.ctx._h, self.id, ctypes.byref(n)))
        return n.value


class Context:
    """One er_ctx: a device, a stream, uploaded frameworks and scratch."""

    def __init__(self, device=0):
        L = _capi.lib()
        h = ctypes.c_void_p()
        st = L.er_ctx_create(int(device), ctypes.byref(h))
        if st != ER_OK:
            raise ErError(st, f"er_ctx_create(device={device}) failed: "
                              f"{L.er_status_string(st).decode()}")
        self._h = h
        self.device = device

    def close(self):
        if self._h:
            _capi.lib().er_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != ER_OK:
            L = _capi.lib()
            raise ErError(st, f"{L.er_status_string(st).decode()}: "
                              f"{L.er_ctx_last_error(self._h).decode()}")

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        self._check(_capi.lib().er_ctx_synchronize(self._h))

    @property
    def stream_ptr(self):
        """The context's cudaStream_t as an int (torch.cuda.ExternalStream(ptr))."""
        v = ctypes.c_void_p()
        self._check(_capi.lib().er_ctx_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    @staticmethod
    def _desc(parts, t_matrix, rep, rc2):
        p = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, 5)
        d = ErFrameworkDesc()
        d.n_atoms = len(p)
        d.atoms = p.ctypes.data
        d.t_matrix[:] = [float(x) for x in np.asarray(t_matrix, dtype=np.float64).reshape(9)]
        d.rep[:] = [int(x) for x in rep]
        d.r_cutoff_squared = float(rc2)
        return d, p

    def upload(self, parts, t_matrix, rep, rc2):
        d, p = self._desc(parts, t_matrix, rep, rc2)
        fid = ctypes.c_int(0)
        self._check(_capi.lib().er_framework_upload(self._h, ctypes.byref(d), ctypes.byref(fid)))
        return Framework(self, fid.value, len(p))

    def upload_many(self, items):
        """items: list of (particles, t_matrix, rep, rc2); one er_framework_upload_many call
        (cell lists built on all host threads)."""
        descs, keep = [], []
        for it in items:
            d, p = self._desc(*it)
            descs.append(d)
            keep.append(p)
        n = len(descs)
        arr = (ErFrameworkDesc * max(n, 1))(*descs)
        ids = (ctypes.c_int * max(n, 1))()
        self._check(_capi.lib().er_framework_upload_many(self._h, arr, n, ids))
        return [Framework(self, ids[i], len(keep[i])) for i in range(n)]

    def grid(self, fw, dims, precision=ER_PREC_NEAR64, f64=False):
        """Host grid (nx, ny, nz) as float32 (or float64)."""
        nx, ny, nz = (int(x) for x in dims)
        out = np.empty((nx, ny, nz), dtype=np.float64 if f64 else np.float32)
        flags = ER_OUT_HOST | (ER_OUT_F64 if f64 else ER_OUT_F32) | precision
        self._check(_capi.lib().er_grid(self._h, fw.id, nx, ny, nz, flags,
                                        out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def grid_device(self, fw, dims, out_ptr, precision=ER_PREC_NEAR64, f64=False):
        """Grid into a caller-owned device buffer (e.g. a torch tensor's data_ptr())."""
        nx, ny, nz = (int(x) for x in dims)
        flags = ER_OUT_DEVICE | (ER_OUT_F64 if f64 else ER_OUT_F32) | precision
        self._check(_capi.lib().er_grid(self._h, fw.id, nx, ny, nz, flags,
                                        ctypes.c_void_p(int(out_ptr))))

    def count_pairs(self, fw, dims):
        """Number of in-cutoff pair terms per grid point (float32 counts)."""
        nx, ny, nz = (int(x) for x in dims)
        out = np.empty((nx, ny, nz), dtype=np.float32)
        self._check(_capi.lib().er_grid(self._h, fw.id, nx, ny, nz,
                                        ER_OUT_HOST | ER_COUNT_PAIRS,
                                        out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def count_pairs_device(self, fw, dims, out_ptr):
        nx, ny, nz = (int(x) for x in dims)
        self._check(_capi.lib().er_grid(self._h, fw.id, nx, ny, nz,
                                        ER_OUT_DEVICE | ER_COUNT_PAIRS,
                                        ctypes.c_void_p(int(out_ptr))))

    def set_timing(self, on=True):
        """Record per-stage device times of er_henry calls (CUDA events)."""
        self._check(_capi.lib().er_ctx_set_timing(self._h, int(bool(on))))

    def henry_timing(self):
        """Stage times (ms) of the last timed er_henry call: bin, sort, energy, reduce."""
        t = _capi.ErHenryTiming()
        self._check(_capi.lib().er_henry_last_timing(self._h, ctypes.byref(t)))
        return {"bin_ms": t.bin_ms, "sort_ms": t.sort_ms, "energy_ms": t.energy_ms,
                "reduce_ms": t.reduce_ms}

    def rcp64_seed_error(self):
        """Largest relative error of the hardware FP64 reciprocal seed."""
        v = ctypes.c_double(0.0)
        self._check(_capi.lib().er_probe_rcp64_seed(self._h, ctypes.byref(v)))
        return v.value

    def fp32_rate(self, seconds=0.2):
        """Measured FP32 FMA issue rate of the device (lane-instructions/s)."""
        v = ctypes.c_double(0.0)
        self._check(_capi.lib().er_probe_fp32_rate(self._h, float(seconds), ctypes.byref(v)))
        return v.value

    def grid_sheet(self, fw, dims, x_index):
        nx, ny, nz = (int(x) for x in dims)
        out = np.empty((ny, nz), dtype=np.float64)
        self._check(_capi.lib().er_grid_sheet(self._h, fw.id, nx, ny, nz, int(x_index),
                                              _dptr(out)))
        return out

    def accessibility(self, fw, dims):
        nx, ny, nz = (int(x) for x in dims)
        out = np.empty((nx, ny, nz), dtype=np.uint8)
        self._check(_capi.lib().er_accessibility(self._h, fw.id, nx, ny, nz,
                                                 _dptr(out, ctypes.c_uint8)))
        return out

    @staticmethod
    def _jobs(jobs):
        arr = (ErGridJob * len(jobs))()
        for k, (fw, dims, ptr) in enumerate(jobs):
            arr[k].fw_id = fw.id
            arr[k].nx, arr[k].ny, arr[k].nz = (int(x) for x in dims)
            arr[k].out_device = int(ptr)
        return arr

    def grid_batch(self, jobs, mode=ER_BATCH_PERSISTENT):
        """jobs: list of (Framework, (nx, ny, nz), device pointer of nx*ny*nz floats)."""
        arr = self._jobs(jobs)
        self._check(_capi.lib().er_grid_batch(self._h, arr, len(jobs), mode))

    def batch_plan(self, jobs, mode=ER_BATCH_PERSISTENT):
        return BatchPlan(self, jobs, mode)

    def henry(self, fw, temperature, n_ins, seed, block_mask=None, want_energies=False):
        m = None
        mnx = mny = mnz = 0
        if block_mask is not None:
            m = np.ascontiguousarray(block_mask, dtype=np.uint8)
            mnx, mny, mnz = m.shape
        res = ErHenryResult()
        en = np.empty(int(n_ins), dtype=np.float32) if want_energies else None
        self._check(_capi.lib().er_henry(
            self._h, fw.id, float(temperature), int(n_ins), int(seed),
            _dptr(m, ctypes.c_uint8) if m is not None else None, mnx, mny, mnz,
            ctypes.byref(res), _dptr(en, ctypes.c_float) if en is not None else None))
        out = {k: getattr(res, k) for k, _ in ErHenryResult._fields_}
        if en is not None:
            out["energies"] = en
        return out

    def henry_device_mask(self, fw, temperature, n_ins, seed, mask_ptr, mask_dims):
        """er_henry with a pocket mask that already lives on the device."""
        mnx, mny, mnz = (int(x) for x in mask_dims)
        res = ErHenryResult()
        self._check(_capi.lib().er_henry(
            self._h, fw.id, float(temperature), int(n_ins), int(seed),
            ctypes.cast(ctypes.c_void_p(int(mask_ptr)), ctypes.POINTER(ctypes.c_uint8)),
            mnx, mny, mnz, ctypes.byref(res), None))
        return {k: getattr(res, k) for k, _ in ErHenryResult._fields_}

    def henry_batch(self, fws, temperature, n_ins, seeds, block_dims=None):
        """er_henry_batch: per framework (optionally) the blocking grid of
        block_dims, its pocket mask, then er_henry with that seed; returns
        (list of result dicts, list of pocket counts)."""
        n = len(fws)
        ids = (ctypes.c_int * max(n, 1))(*[f.id for f in fws])
        sd = (ctypes.c_uint64 * max(n, 1))(*[int(s) for s in seeds])
        res = (ErHenryResult * max(n, 1))()
        npk = (ctypes.c_int * max(n, 1))()
        bx, by, bz = (int(x) for x in block_dims) if block_dims is not None else (0, 0, 0)
        self._check(_capi.lib().er_henry_batch(self._h, ids, n, float(temperature), int(n_ins),
                                               sd, bx, by, bz, res, npk))
        out = [{k: getattr(res[i], k) for k, _ in ErHenryResult._fields_} for i in range(n)]
        return out, [npk[i] for i in range(n)]

    def block_pockets(self, grid, temperature, want_segments=False):
        """FindAndBlockPockets on a host float64 grid; returns (grid copy, n_pockets[, seg])."""
        g = np.array(grid, dtype=np.float64, copy=True, order="C")
        nx, ny, nz = g.shape
        n = ctypes.c_int(0)
        seg = np.empty(g.shape, dtype=np.int32) if want_segments else None
        self._check(_capi.lib().er_block_pockets(
            self._h, _dptr(g), nx, ny, nz, float(temperature), ctypes.byref(n),
            _dptr(seg, ctypes.c_int) if seg is not None else None))
        if want_segments:
            return g, n.value, seg
        return g, n.value

    def grid_interp(self, grid_ptr, dims, pts, f64=False):
        """GCMC guest-framework energies at fractional points (n, 3) by trilinear
        lookup in a device grid (float, or double with f64=True); host in/out."""
        q = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        out = np.empty(len(q), dtype=np.float64)
        _grid_interp(self, grid_ptr, dims, q.ctypes.data, len(q), out.ctypes.data, f64)
        return out

    def grid_interp_device(self, grid_ptr, dims, pts_ptr, n, out_ptr, f64=False):
        """As grid_interp with points and results in device memory."""
        _grid_interp(self, grid_ptr, dims, pts_ptr, n, out_ptr, f64)

    def block_pockets_device(self, grid_ptr, dims, temperature, mask_ptr):
        nx, ny, nz = (int(x) for x in dims)
        n = ctypes.c_int(0)
        self._check(_capi.lib().er_block_pockets_device(
            self._h, ctypes.c_void_p(int(grid_ptr)), nx, ny, nz, float(temperature),
            ctypes.c_void_p(int(mask_ptr)), ctypes.byref(n)))
        return n.value


def _grid_interp(ctx, grid_ptr, dims, pts_ptr, n, out_ptr, f64):
    nx, ny, nz = (int(x) for x in dims)
    ctx._check(_capi.lib().er_grid_interp(
        ctx._h, ctypes.c_void_p(int(grid_ptr)), nx, ny, nz, ER_INTERP_GRID_F64 if f64 else 0,
        ctypes.cast(ctypes.c_void_p(int(pts_ptr)), ctypes.POINTER(ctypes.c_double)), int(n),
        ctypes.cast(ctypes.c_void_p(int(out_ptr)), ctypes.POINTER(ctypes.c_double))))


class BatchPlan:
    """A fixed work queue replayed as a CUDA graph (er_batch_plan_*)."""

    def __init__(self, ctx, jobs, mode):
        self.ctx = ctx
        self._keep = jobs
        arr = Context._jobs(jobs)
        h = ctypes.c_void_p()
        ctx._check(_capi.lib().er_batch_plan_create(ctx._h, arr, len(jobs), mode,
                                                    ctypes.byref(h)))
        self._h = h

    def run(self):
        self.ctx._check(_capi.lib().er_batch_plan_run(self._h))

    @property
    def launches(self):
        n = ctypes.c_int(0)
        self.ctx._check(_capi.lib().er_batch_plan_launches(self._h, ctypes.byref(n)))
        return n.value

    def tile(self, job):
        """Points per thread (4 or 8) of the kernel variant used for job `job`."""
        n = ctypes.c_int(0)
        self.ctx._check(_capi.lib().er_batch_plan_tile(self._h, int(job), ctypes.byref(n)))
        return n.value

    def close(self):
        if self._h:
            _capi.lib().er_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
