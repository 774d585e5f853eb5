"""Python side of the request server (er_server_*, include/emptyroom_b200.h).

`Server(ctx, budget_bytes, slots)` accepts grid and Henry jobs from any
thread; `slots=1` is the plain one-job-at-a-time loop. `run_stream` replays a
timed arrival schedule against a server and returns per-job latencies.
"""
from __future__ import annotations

import ctypes
import threading
import time

import numpy as np

from . import ErFrameworkDesc, ErHenryResult, _capi
from ._capi import ErJob, ErJobStatus

ER_JOB_GRID = 1
ER_JOB_HENRY = 2


class ServerError(RuntimeError):
    pass


def framework_desc(parts, t_matrix, rep, rc2):
    """An er_framework_desc that owns its particle array (keep the object alive)."""
    p = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, 5)
    d = ErFrameworkDesc()
    d.n_atoms = len(p)
    d.atoms = p.ctypes.data
    d.t_matrix[:] = [float(x) for x in np.asarray(t_matrix, dtype=np.float64).reshape(9)]
    d.rep[:] = [int(x) for x in rep]
    d.r_cutoff_squared = float(rc2)
    d._keep = p
    return d


class Server:
    def __init__(self, ctx, budget_bytes, slots):
        self.ctx = ctx
        h = ctypes.c_void_p()
        st = _capi.lib().er_server_create(ctx.handle, int(budget_bytes), int(slots),
                                          ctypes.byref(h))
        if st != 0:
            raise ServerError(f"er_server_create failed: {st}")
        self._h = h
        self._keep = {}

    def submit_grid(self, fw_key, desc, dims, out_host=None):
        j = ErJob()
        j.kind = ER_JOB_GRID
        j.fw_key = int(fw_key)
        j.desc = ctypes.cast(ctypes.pointer(desc), ctypes.c_void_p)
        j.nx, j.ny, j.nz = (int(x) for x in dims)
        j.grid_out_host = out_host if out_host is not None else None
        return self._submit(j, desc)

    def submit_henry(self, fw_key, desc, temperature, n_ins, seed):
        j = ErJob()
        j.kind = ER_JOB_HENRY
        j.fw_key = int(fw_key)
        j.desc = ctypes.cast(ctypes.pointer(desc), ctypes.c_void_p)
        j.temperature = float(temperature)
        j.n_insertions = int(n_ins)
        j.seed = int(seed)
        return self._submit(j, desc)

    def _submit(self, j, desc):
        t = ctypes.c_uint64(0)
        st = _capi.lib().er_server_submit(self._h, ctypes.byref(j), ctypes.byref(t))
        if st != 0:
            raise ServerError(f"er_server_submit failed: {st}")
        self._keep[t.value] = desc
        return t.value

    def wait(self, ticket, timeout=600.0):
        s = ErJobStatus()
        st = _capi.lib().er_server_wait(self._h, int(ticket), float(timeout), ctypes.byref(s))
        if st == 6:
            raise TimeoutError(f"job {ticket} still running")
        if st != 0:
            raise ServerError(f"er_server_wait failed: {st}")
        return _status_dict(s)

    def poll(self, ticket):
        s = ErJobStatus()
        st = _capi.lib().er_server_poll(self._h, int(ticket), ctypes.byref(s))
        if st != 0:
            raise ServerError(f"er_server_poll failed: {st}")
        return _status_dict(s)

    def grid_ptr(self, ticket):
        p = ctypes.c_void_p()
        st = _capi.lib().er_server_grid(self._h, int(ticket), ctypes.byref(p))
        if st != 0:
            raise ServerError(f"grid of job {ticket} not resident")
        return p.value

    def now(self):
        return _capi.lib().er_server_now(self._h)

    @property
    def device_bytes(self):
        n = ctypes.c_size_t(0)
        _capi.lib().er_server_bytes(self._h, ctypes.byref(n))
        return n.value

    def close(self):
        if self._h:
            _capi.lib().er_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _status_dict(s):
    d = {k: getattr(s, k) for k, _ in ErJobStatus._fields_ if k != "henry"}
    d["henry"] = {k: getattr(s.henry, k) for k, _ in ErHenryResult._fields_}
    d["latency_s"] = s.finish_s - s.submit_s if s.done else None
    return d


def run_stream(server, schedule):
    """schedule: list of (arrival_s, submit_fn) sorted by arrival; submit_fn(server)
    returns a ticket. Submits each job at its arrival time (server clock) from
    this thread, then waits for all. Returns the list of statuses in order."""
    t_start = server.now()
    tickets = []
    for arrival, fn in schedule:
        while True:
            dt = t_start + arrival - server.now()
            if dt <= 0:
                break
            time.sleep(min(dt, 0.002) if dt > 0.0005 else 0)
        tickets.append(fn(server))
    return [server.wait(t) for t in tickets]
