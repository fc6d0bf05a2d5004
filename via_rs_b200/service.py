"""Python binding of the continuous-batching answer service (via_service_* in include/via_gpu.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .server import Server, check


class ServiceConfig(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_uint32), ("max_batch", ctypes.c_uint32), ("hbm_budget", ctypes.c_uint64),
                ("max_pending", ctypes.c_uint32), ("warm", ctypes.c_uint32), ("autotune", ctypes.c_uint32),
                ("tune_cache", ctypes.c_char_p)]


class ServiceStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("units", ctypes.c_uint64), ("lanes", ctypes.c_uint32),
                ("batch_cap", ctypes.c_uint32), ("max_in_flight", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_batch", ctypes.c_double),
                ("answers_per_s", ctypes.c_double)]


def _bind():
    L = _lib.lib()
    if getattr(L, "_service_bound", False):
        return L
    vp = ctypes.c_void_p
    L.via_service_create.restype = ctypes.c_int
    L.via_service_create.argtypes = [vp, ctypes.POINTER(ServiceConfig), ctypes.POINTER(vp)]
    L.via_service_submit.restype = ctypes.c_int
    L.via_service_submit.argtypes = [vp, vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    L.via_service_poll.restype = ctypes.c_int
    L.via_service_poll.argtypes = [vp, ctypes.c_uint64, vp, vp, ctypes.POINTER(ctypes.c_int)]
    L.via_service_wait.restype = ctypes.c_int
    L.via_service_wait.argtypes = [vp, ctypes.c_uint64, vp, vp, ctypes.c_uint32]
    L.via_service_stats_get.restype = ctypes.c_int
    L.via_service_stats_get.argtypes = [vp, ctypes.POINTER(ServiceStats)]
    L.via_server_workspace_bytes.restype = ctypes.c_uint64
    L.via_server_workspace_bytes.argtypes = [vp, ctypes.c_uint64]
    L.via_service_stats_reset.restype = ctypes.c_int
    L.via_service_stats_reset.argtypes = [vp]
    L.via_service_latencies.restype = ctypes.c_uint64
    L.via_service_latencies.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64]
    L.via_service_tuning.restype = ctypes.c_uint64
    L.via_service_tuning.argtypes = [vp, ctypes.POINTER(_lib.ScanTuning), ctypes.c_uint64]
    L.via_service_destroy.restype = None
    L.via_service_destroy.argtypes = [vp]
    L._service_bound = True
    return L


def workspace_bytes(server: Server, max_queries: int) -> int:
    """Device bytes of one service lane's workspace for batches of max_queries queries."""
    return int(_bind().via_server_workspace_bytes(server._h, max_queries))


class Service:
    """Continuous batching over one Server: submit() queues a request (one VIA-C
    query, or T = n2 / n_rec queries for a VIA-B server) and returns a ticket;
    poll()/wait() return its (mask, body) answer."""

    def __init__(self, server: Server, lanes: int = 2, max_batch: int = 64, hbm_budget: int = 0,
                 max_pending: int = 0, warm: bool = False, autotune: bool = False, tune_cache: str | None = None):
        self.server = server
        self.prm = server.prm
        L = _bind()
        cfg = ServiceConfig(lanes, max_batch, hbm_budget, max_pending, 1 if warm else 0, 1 if autotune else 0,
                            tune_cache.encode() if tune_cache else None)
        h = ctypes.c_void_p()
        check(L.via_service_create(server._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def latencies(self) -> np.ndarray:
        """Submit-to-completion latencies (ms) of the requests completed since
        creation or the last reset, in completion order."""
        L = _bind()
        n = int(L.via_service_latencies(self._h, None, 0))
        out = np.zeros(max(1, n), dtype=np.float64)
        n = int(L.via_service_latencies(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out[:n]

    def tuning(self) -> list:
        """The scan autotuner's choices made at creation (empty without autotune)."""
        L = _bind()
        n = int(L.via_service_tuning(self._h, None, 0))
        out = (_lib.ScanTuning * max(1, n))()
        L.via_service_tuning(self._h, out, n)
        return [out[i].as_dict() for i in range(n)]

    def submit(self, query) -> int:
        q = np.ascontiguousarray(query, dtype=np.uint64).reshape(-1)
        t = ctypes.c_uint64()
        check(_bind().via_service_submit(self._h, q.ctypes.data_as(ctypes.c_void_p), self.prm.n_lwe,
                                         ctypes.byref(t)))
        return t.value

    def _bufs(self):
        return np.zeros(self.prm.n2, dtype=np.uint64), np.zeros(self.prm.n2, dtype=np.uint64)

    def poll(self, ticket: int):
        m, b = self._bufs()
        done = ctypes.c_int()
        check(_bind().via_service_poll(self._h, ticket, m.ctypes.data_as(ctypes.c_void_p),
                                       b.ctypes.data_as(ctypes.c_void_p), ctypes.byref(done)))
        return (m, b) if done.value else None

    def wait(self, ticket: int, timeout_ms: int = 120000):
        m, b = self._bufs()
        check(_bind().via_service_wait(self._h, ticket, m.ctypes.data_as(ctypes.c_void_p),
                                       b.ctypes.data_as(ctypes.c_void_p), timeout_ms))
        return m, b

    def stats(self) -> dict:
        st = ServiceStats()
        check(_bind().via_service_stats_get(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServiceStats._fields_ if f != "reserved"}

    def reset_stats(self) -> None:
        check(_bind().via_service_stats_reset(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _bind().via_service_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
