"""The client side on the GPU (include/via_gpu.h via_client_*): Client::query and
Client::recover of the reference's via-client (crates/via-client/src), bit-exact
with its PRG and samplers, for load generation and many-query clients."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import Params, ViaParams
from .server import check

ERR_TERNARY = 0
ERR_BOUNDED_UNIFORM = 1


def _bind():
    L = _lib.lib()
    if getattr(L, "_client_bound", False):
        return L
    vp = ctypes.c_void_p
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.via_client_create.restype = ctypes.c_int
    L.via_client_create.argtypes = [ctypes.POINTER(ViaParams), u64p, u64p, ctypes.c_uint32, ctypes.c_uint32,
                                    ctypes.POINTER(vp)]
    L.via_client_destroy.restype = None
    L.via_client_destroy.argtypes = [vp]
    L.via_client_queries.restype = ctypes.c_int
    L.via_client_queries.argtypes = [vp, u64p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint32, u64p]
    L.via_client_queries_dev.restype = ctypes.c_int
    L.via_client_queries_dev.argtypes = [vp, u64p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint32, vp, vp]
    L.via_client_recover.restype = ctypes.c_int
    L.via_client_recover.argtypes = [vp, u64p, u64p, ctypes.c_uint64, u64p]
    L._client_bound = True
    return L


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


class Client:
    """Client with secret keys sk1 (nl * n1 residues at q1) and sk2 (n2 at q3)."""

    def __init__(self, prm: Params, sk1, sk2, err_kind: int = ERR_TERNARY, err_bound: int = 0):
        L = _bind()
        self.prm = prm
        cp = prm.to_c()
        s1, s2 = _u64(sk1), _u64(sk2)
        h = ctypes.c_void_p()
        check(L.via_client_create(ctypes.byref(cp), _p(s1), _p(s2), err_kind, err_bound, ctypes.byref(h)))
        self._h = h

    @staticmethod
    def _seeds(seeds) -> tuple:
        seeds = [bytes(s) for s in seeds]
        n = len(seeds[0])
        if any(len(s) != n for s in seeds):
            raise ValueError("every seed must have the same length")
        return b"".join(seeds), n

    def queries(self, indices, seeds) -> np.ndarray:
        """Client::query for each (index, seed): [count][n_lwe * lwe_len]."""
        prm = self.prm
        idx = _u64(indices).reshape(-1)
        blob, n = self._seeds(seeds)
        out = np.zeros((idx.size, prm.n_lwe * prm.lwe_len), dtype=np.uint64)
        check(_bind().via_client_queries(self._h, _p(idx), idx.size, blob, n, _p(out)))
        return out

    def query(self, index: int, seed: bytes) -> np.ndarray:
        return self.queries([index], [seed])[0]

    def queries_dev(self, indices, seeds, out_ptr: int, stream: int = 0) -> None:
        idx = _u64(indices).reshape(-1)
        blob, n = self._seeds(seeds)
        check(_bind().via_client_queries_dev(self._h, _p(idx), idx.size, blob, n, ctypes.c_void_p(out_ptr),
                                             ctypes.c_void_p(stream)))

    def recover_many(self, masks, bodies) -> np.ndarray:
        prm = self.prm
        m = _u64(masks).reshape(-1, prm.n2)
        b = _u64(bodies).reshape(-1, prm.n2)
        out = np.zeros_like(m)
        check(_bind().via_client_recover(self._h, _p(m), _p(b), m.shape[0], _p(out)))
        return out

    def recover(self, mask, body) -> np.ndarray:
        return self.recover_many(mask, body)[0]

    def recover_batch(self, mask, body) -> list:
        """Client::recover_batch: record t of a VIA-B answer is every T-th coefficient from t."""
        plain = self.recover(mask, body)
        stride = self.prm.n2 // self.prm.n_rec
        return [plain[t::stride] for t in range(stride)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            _bind().via_client_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
