"""Mixed serving over one database: VIA-C queries and VIA-B batches side by side.

The reference serves each record degree from its own Server (and its own copy
of the prepared database); a VIA-B request of m indices is padded by the client
to the batch size T = n2 / n3 of the server it goes to (cli/client.rs:256-300).
Here one prepared database in HBM is read through one view per record degree
(via_server_view), and each view has its own continuous-batching service with
a share of the HBM budget. A VIA-B request of m indices goes to the smallest
power-of-two batch size T >= m. Requests of one kind are batched per database
scan; the services' lanes overlap on the GPU.
"""
from __future__ import annotations

import os
import tempfile

import numpy as np

from .server import Server
from .service import Service, workspace_bytes

# VIA-B batch sizes T = n2 / n_rec: every power of two the record-fit rule
# admits at n2 = 512 (crates/via-protocol/src/presets.rs:170-176; the repack is
# generic over T, crates/via-primitives/src/conversion/repack.rs:331-397).
POW2_BATCH_SIZES = (2, 4, 8, 16, 32, 64, 128, 256)


def via_b_route(m: int, batch_sizes=POW2_BATCH_SIZES) -> int:
    """The smallest VIA-B batch size T that holds a request of m indices."""
    for t in sorted(batch_sizes):
        if m <= t:
            return t
    raise ValueError(f"a VIA-B request of {m} indices exceeds the largest batch size {max(batch_sizes)}")


def _lane_queries(route, max_batch: int) -> int:
    """Queries a lane of this route's service should hold: max_batch VIA-C
    queries, or a VIA-B batch of T queries (at least 16, at most max_batch)."""
    return max_batch if route == "c" else min(max(route, 16), max_batch)


class MixedService:
    """Routes: "c" (VIA-C, one query per request) and one VIA-B route per batch
    size T (records of degree n2 / T, T queries per request).

    hbm_budget (bytes, 0 = unbounded) is split over the routes in proportion to
    the workspace each route's lanes want (`shares` overrides the split). Every
    view reads the same database planes, so the scan tiles the first service
    tunes are reused by the others through one tuning cache file."""

    def __init__(self, base: Server, batch_sizes=POW2_BATCH_SIZES, lanes: int = 2, hbm_budget: int = 0,
                 shares: dict | None = None, max_batch: int = 64, warm: bool = True, autotune: bool = True,
                 keys: dict | None = None):
        prm = base.prm
        if prm.n_rec != prm.n2:
            raise ValueError("the base server must be the VIA-C view (n_rec = n2)")
        self.base = base
        self.servers = {"c": base}
        for t in batch_sizes:
            self.servers[t] = base.view(prm.n2 // t, (keys or {}).get(t))
        if shares is None:
            want = {k: lanes * workspace_bytes(srv, _lane_queries(k, max_batch)) for k, srv in self.servers.items()}
            total = sum(want.values())
            shares = {k: v / total for k, v in want.items()}
        self.shares = shares
        fd, self._tune_cache = tempfile.mkstemp(prefix="via-mixed-tiles-", suffix=".txt")
        os.close(fd)
        self.services = {}
        for k, srv in self.servers.items():
            budget = int(hbm_budget * shares[k]) if hbm_budget else 0
            self.services[k] = Service(srv, lanes=lanes, max_batch=max_batch, hbm_budget=budget, warm=warm,
                                       autotune=autotune, tune_cache=self._tune_cache)

    def params(self, route):
        return self.servers[route].prm

    def submit(self, route, queries) -> tuple:
        """route "c" with one query, or T (a VIA-B batch size) with T queries."""
        return route, self.services[route].submit(queries)

    def wait(self, handle, timeout_ms: int = 600000):
        route, ticket = handle
        return self.services[route].wait(ticket, timeout_ms)

    def latencies(self) -> dict:
        return {k: s.latencies() for k, s in self.services.items()}

    def stats(self) -> dict:
        return {k: s.stats() for k, s in self.services.items()}

    def reset_stats(self) -> None:
        for s in self.services.values():
            s.reset_stats()

    def close_services(self) -> None:
        """Stops the services and frees their lanes; the views stay usable."""
        for s in self.services.values():
            s.close()
        self.services = {}

    def close(self) -> None:
        self.close_services()
        for k, srv in self.servers.items():
            if k != "c":
                srv.close()
        self.servers = {"c": self.base}
        if getattr(self, "_tune_cache", None):
            try:
                os.unlink(self._tune_cache)
            except OSError:
                pass
            self._tune_cache = None


def poisson_mix(n: int, rate_hz: float, seed: int, via_c_fraction: float = 0.5, max_indices: int = 256):
    """A seeded arrival stream: (gap_s, kind, m) with kind "c" (one query) or "b"
    (a VIA-B request of m indices, m log-uniform in [1, max_indices])."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        gap = float(rng.exponential(1.0 / rate_hz))
        if rng.random() < via_c_fraction:
            out.append((gap, "c", 1))
        else:
            m = int(np.floor(np.exp(rng.uniform(0.0, np.log(max_indices + 1)))))
            out.append((gap, "b", max(1, min(max_indices, m))))
    return out
