"""Mixed serving over one database: VIA-C queries and VIA-B batches side by side.

The reference serves each record degree from its own Server (and its own copy
of the prepared database); a VIA-B request of m indices is padded by the client
to the batch size T = n2 / n3 of the server it goes to (cli/client.rs:256-300).
Here one prepared database in HBM is read through one view per record degree
(via_server_view), and each view has its own continuous-batching service with
a share of the HBM budget. Requests of one kind are batched per database scan;
the services' lanes overlap on the GPU.
"""
from __future__ import annotations

import numpy as np

from .server import Server
from .service import Service


def via_b_route(m: int, batch_sizes=(8, 256)) -> int:
    """The smallest VIA-B batch size T that holds a request of m indices."""
    for t in sorted(batch_sizes):
        if m <= t:
            return t
    raise ValueError(f"a VIA-B request of {m} indices exceeds the largest batch size {max(batch_sizes)}")


class MixedService:
    """Routes: "c" (VIA-C, one query per request) and one VIA-B route per batch
    size T (records of degree n2 / T, T queries per request)."""

    def __init__(self, base: Server, batch_sizes=(8, 256), lanes: int = 2, hbm_budget: int = 0,
                 shares: dict | None = None, max_batch: int = 64, warm: bool = True, autotune: bool = True,
                 keys: dict | None = None):
        prm = base.prm
        if prm.n_rec != prm.n2:
            raise ValueError("the base server must be the VIA-C view (n_rec = n2)")
        self.base = base
        self.servers = {"c": base}
        for t in batch_sizes:
            self.servers[t] = base.view(prm.n2 // t, (keys or {}).get(t))
        shares = shares or {k: 1.0 / len(self.servers) for k in self.servers}
        self.services = {}
        for k, srv in self.servers.items():
            budget = int(hbm_budget * shares[k]) if hbm_budget else 0
            self.services[k] = Service(srv, lanes=lanes, max_batch=max_batch, hbm_budget=budget, warm=warm,
                                       autotune=autotune)

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
