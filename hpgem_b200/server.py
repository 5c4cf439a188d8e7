"""Serving loop (hgg_server_* of the C ABI): continuous batching of solves.

Requests are admitted in arrival order while their device footprint fits the
budget, keep their state on the device, and advance together with every other
running request (one launch per RK stage and kernel class); requests that
arrive while others run join at the next chunk boundary.  The GPU thread keeps
two chunks of steps in flight; finished solutions are copied back and freed on
a retire thread.
"""
import ctypes
import threading

import numpy as np

from . import _native


class Server:
    def __init__(self, budget_bytes, max_chunk=25, setup_threads=4, capacity=4096):
        self._lib = _native.load()
        raw = ctypes.c_void_p()
        _native.check_server(self._lib.hgg_server_start(int(budget_bytes), int(max_chunk), int(setup_threads),
                                                        int(capacity), ctypes.byref(raw)))
        self._raw = raw
        self._keep = {}  # request id -> objects the native side still points to
        self._lock = threading.Lock()
        self._lengths = {}

    def _check(self, code):
        return _native.check_server(code, self._raw)

    def submit(self, description, order, physics, params, dt, nsteps, u0=None, initial=None,
               tableau="RK4_4", precision=_native.PRECISION_FP64, n_vars=1):
        """Queues a solve.  The initial condition is either coefficients `u0` (hpGEM
        order) or a function initial(x[n, dim]) -> [n] or [n, n_vars] that the server
        projects; returns the request id."""
        code = {"advection": _native.PHYSICS_ADVECTION, "wave": _native.PHYSICS_WAVE,
                "wave_upwind": _native.PHYSICS_WAVE_UPWIND}[physics]
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        keep = [p]
        u0p, n_u0 = None, 0
        if u0 is not None:
            a = np.ascontiguousarray(np.asarray(u0, dtype=np.float64).reshape(-1))
            keep.append(a)
            u0p, n_u0 = ctypes.c_void_p(a.ctypes.data), a.size
        cb = _native.INITIAL_FN()
        if initial is not None:
            def fn(xyz, n, dim, values, user, _f=initial, _v=int(n_vars)):
                x = np.ctypeslib.as_array(xyz, shape=(n, dim))
                out = np.ctypeslib.as_array(values, shape=(n, _v))
                out[...] = np.asarray(_f(x), dtype=np.float64).reshape(n, _v)
            cb = _native.INITIAL_FN(fn)
            keep.append(cb)
        rid = ctypes.c_int64()
        self._check(self._lib.hgg_server_submit(self._raw, description.encode(), int(order), code,
                                                ctypes.c_void_p(p.ctypes.data), p.size, tableau.encode(),
                                                int(precision), u0p, n_u0, cb, None, float(dt), int(nsteps),
                                                ctypes.byref(rid)))
        with self._lock:
            self._keep[rid.value] = keep
        return rid.value

    def poll(self, rid, wait=False, result=True):
        """(done, solution or None, latency in seconds or None)."""
        lat = ctypes.c_double()
        code = self._check(self._lib.hgg_server_poll(self._raw, int(rid), 1 if wait else 0, None, 0,
                                                     ctypes.byref(lat)))
        if code == 0:
            return False, None, None
        out = None
        if result:
            n = int(self._lib.hgg_server_result_length(self._raw, int(rid)))
            out = np.empty(n)
            self._check(self._lib.hgg_server_poll(self._raw, int(rid), 0, ctypes.c_void_p(out.ctypes.data), n,
                                                  ctypes.byref(lat)))
        with self._lock:
            self._keep.pop(int(rid), None)
        return True, out, lat.value

    def times(self, rid):
        t = np.zeros(4)
        self._check(self._lib.hgg_server_times(self._raw, int(rid), ctypes.c_void_p(t.ctypes.data)))
        return t

    def release(self, rid):
        self._check(self._lib.hgg_server_release(self._raw, int(rid)))

    def stats(self):
        st = np.zeros(4, dtype=np.int64)
        self._check(self._lib.hgg_server_stats(self._raw, ctypes.c_void_p(st.ctypes.data)))
        t = np.zeros(8)
        self._check(self._lib.hgg_server_timing(self._raw, ctypes.c_void_p(t.ctypes.data)))
        return dict(completed=int(st[0]), dof_updates=int(st[1]), chunks=int(st[2]), reserved_bytes=int(st[3]),
                    gpu_thread_step_s=float(t[0]), gpu_thread_members_s=float(t[1]),
                    gpu_thread_idle_s=float(t[2]), retire_thread_s=float(t[3]), device_chunk_s=float(t[4]),
                    gpu_thread_join_s=float(t[5]), gpu_thread_tables_s=float(t[6]),
                    retire_copyback_s=float(t[7]))

    def stop(self):
        if self._raw:
            rc = self._lib.hgg_server_stop(self._raw)
            self._raw = None
            self._keep.clear()
            _native.check_server(rc, None)

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
