"""Served requests: a stream of independent energy+force / MD requests of mixed sizes on one GPU (ix_server_*).

The scheduling runs in the library's native worker thread: admission by a device-memory budget, continuous batching
(periodic systems as contexts on their own streams, small non-periodic systems gathered into batched cohorts), and
results unpacked from pinned staging as each request's last step completes.  This class only describes requests and
collects results.

The requests run on many CUDA streams at once; their kernels overlap on the device only as far as its hardware work
queues keep the streams apart.  Set CUDA_DEVICE_MAX_CONNECTIONS=32 in the environment before CUDA starts in the
process (the default 8 queues leave a small request waiting behind other requests' work: on the 20,000-request
stream, p50 latency 172 ms with 8 queues, 6 ms with 32).  With 32 queues, two or three worker threads (`threads`)
launch requests in parallel without contending in the driver (on that stream, 441 requests/s with one thread, 549 with
three).
"""
import ctypes

import numpy as np

from . import _capi
from .context import describe_forces
from .forces import OpenMMException


class Result:
    __slots__ = ("id", "positions", "velocities", "forces", "term_energies", "latency", "status", "error")

    def __init__(self, **kw):
        for k in self.__slots__:
            setattr(self, k, kw.get(k))

    @property
    def energy(self):
        return float(self.term_energies.sum())


class Server:
    def __init__(self, device=0, budget_bytes=120e9, max_running=256, small_atoms=1024, max_cohort=512,
                 window_seconds=200e-6, threads=1):
        self._lib = _capi.lib()
        self._srv = ctypes.c_void_p()
        rc = self._lib.ix_server_create(int(device), float(budget_bytes), int(max_running), int(threads),
                                        ctypes.byref(self._srv))
        if rc != _capi.IX_OK:
            self._srv = ctypes.c_void_p()
            raise OpenMMException(self._lib.ix_server_last_error(None).decode())
        self._check(self._lib.ix_server_set_batching(self._srv, int(small_atoms), int(max_cohort),
                                                     float(window_seconds)))
        self._sizes = {}
        self._templates = {}

    def _check(self, rc):
        if rc != _capi.IX_OK:
            raise OpenMMException(self._lib.ix_server_last_error(self._srv).decode())

    class _Recorder:
        """Stands in for the library while describe_forces runs once per System: records the ix_add_* calls so that
        each request replays them without converting the System again."""

        def __init__(self):
            self.calls = []

        def __getattr__(self, name):
            def record(handle, *args):
                self.calls.append((name, args))
                return _capi.IX_OK
            return record

    def _template(self, system):
        t = self._templates.get(id(system))
        if t is None or t[0] is not system:
            rec, keep = self._Recorder(), []
            describe_forces(rec, None, system, lambda rc: None, keep)
            n = system.getNumParticles()
            box = _capi.arr(np.asarray(system.getDefaultPeriodicBoxVectors()).reshape(9), np.float64)
            mass = _capi.arr([system.getParticleMass(i) for i in range(n)], np.float64)
            t = (system, n, box, mass, rec.calls, keep)
            self._templates[id(system)] = t
        return t

    def submit(self, system, positions, velocities=None, steps=0, dt=0.001, parameters=None, list_capacity=None):
        """Queue `steps` velocity-Verlet steps of `dt` ps of `system` from the given state (0 steps: one energy+force
        evaluation).  Masses come from the System.  list_capacity: (pair tiles, three-body entries per site) of the
        request's neighbor lists at admission (ix_set_list_capacity; None = estimated).  Returns the request id."""
        L = self._lib
        _, n, box, mass, calls, _ = self._template(system)
        req = ctypes.c_void_p()
        if L.ix_request_create(n, _capi.ptr(box), ctypes.byref(req)) != _capi.IX_OK:
            raise OpenMMException(L.ix_last_error(None).decode())
        owned = True
        try:
            def check(rc):
                if rc != _capi.IX_OK:
                    raise OpenMMException(L.ix_last_error(req).decode())
            for name, args in calls:
                check(getattr(L, name)(req, *args))
            for k, v in (parameters or {}).items():
                check(L.ix_set_parameter(req, k.encode(), float(v)))
            if list_capacity is not None:
                check(L.ix_set_list_capacity(req, int(list_capacity[0]), int(list_capacity[1])))
            pos = _capi.arr(np.asarray(positions, dtype=np.float64).reshape(n, 3), np.float64)
            vel = None if velocities is None else _capi.arr(np.asarray(velocities).reshape(n, 3), np.float64)
            check(L.ix_request_set_state(req, _capi.ptr(pos), _capi.ptr(vel), _capi.ptr(mass)))
            rid = ctypes.c_longlong()
            self._check(L.ix_server_submit(self._srv, req, int(steps), float(dt), ctypes.byref(rid)))
            owned = False
        finally:
            if owned:
                L.ix_ctx_destroy(req)
        self._sizes[rid.value] = n
        return rid.value

    def poll(self, max_ids=4096):
        ids = np.zeros(max_ids, dtype=np.int64)
        count = ctypes.c_int()
        self._check(self._lib.ix_server_poll(self._srv, max_ids, _capi.ptr(ids), ctypes.byref(count)))
        return ids[:count.value].tolist()

    def wait(self, timeout=1.0, max_ids=4096):
        ids = np.zeros(max_ids, dtype=np.int64)
        count = ctypes.c_int()
        self._check(self._lib.ix_server_wait(self._srv, float(timeout), max_ids, _capi.ptr(ids), ctypes.byref(count)))
        return ids[:count.value].tolist()

    def result(self, rid):
        """The result of a completed request (then released by the server)."""
        n = self._sizes.pop(rid)
        pos, vel, frc, en = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(4)
        lat = ctypes.c_double()
        rc = self._lib.ix_server_result(self._srv, int(rid), _capi.ptr(pos), _capi.ptr(vel), _capi.ptr(frc),
                                        _capi.ptr(en), ctypes.byref(lat))
        err = None if rc == _capi.IX_OK else self._lib.ix_server_last_error(self._srv).decode()
        return Result(id=rid, positions=pos, velocities=vel, forces=frc, term_energies=en, latency=lat.value,
                      status=rc, error=err)

    def run_all(self, timeout=600.0):
        """Wait for every submitted request; returns {id: Result}."""
        out = {}
        while self._sizes.keys() - out.keys():
            ids = self.wait(timeout)
            if not ids:
                raise OpenMMException("timed out waiting for requests")
            for rid in ids:
                out[rid] = self.result(rid)
        return out

    def stats(self):
        s = _capi.ServerStats()
        self._check(self._lib.ix_server_stats_get(self._srv, ctypes.byref(s)))
        out = {k: getattr(s, k) for k, _ in s._fields_}
        out["worker_seconds"] = dict(zip(("context_setup", "context_enqueue", "cohort_build", "cohort_enqueue",
                                          "teardown", "event_checks", "admission", "idle", "pinned_staging",
                                          "device_setup", "state_uploads", "step_launches"),
                                         list(s.worker_seconds)))
        return out

    def close(self):
        if getattr(self, "_srv", None) and self._srv.value:
            self._lib.ix_server_destroy(self._srv)
            self._srv = ctypes.c_void_p()

    def __del__(self):
        self.close()
