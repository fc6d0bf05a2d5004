"""Host-side mirror of via-server's `Server` (crates/via-server/src/answer.rs:423-603).

    server = Server.setup(params, keys, records)     # Server::setup
    mask, body = server.answer(query)                 # Server::answer

Errors mirror `via_protocol::ViaError` (crates/via-protocol/src/error.rs:20-64):
the reference returns `Err(ViaError::DimMismatch(..))` /
`Err(ViaError::QueryLengthMismatch{..})`; here the same conditions raise
`DimMismatch` / `QueryLengthMismatch`.
"""
import ctypes

import numpy as np

from . import _lib
from .params import Params

VIA_RECORDS_U64 = 0
VIA_RECORDS_NIBBLE = 1


class ViaError(RuntimeError):
    code = -1


class SetupNotComplete(ViaError):
    code = 1


class IndexOutOfRange(ViaError):
    code = 2


class QueryLengthMismatch(ViaError):
    code = 3


class BufferTooShort(ViaError):
    code = 4


class UnknownFormatTag(ViaError):
    code = 5


class DimMismatch(ViaError):
    code = 7


class DeviceError(ViaError):
    """A device-side failure (allocation, CUDA call, bounded wait)."""


_BY_CODE = {c.code: c for c in (SetupNotComplete, IndexOutOfRange, QueryLengthMismatch, BufferTooShort,
                               UnknownFormatTag, DimMismatch)}


def check(rc: int) -> None:
    if rc != 0:
        msg = _lib.lib().via_last_error().decode()
        cls = _BY_CODE.get(rc, DeviceError)
        err = cls(f"[{rc}] {msg}")
        err.code = rc
        raise err


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


class PublicKeys:
    """The client's public keys in include/via_gpu.h wire layout."""

    def __init__(self, cascade_key, conv_key, rsk):
        self.cascade_key = _u64(cascade_key)
        self.conv_key = _u64(conv_key)
        self.rsk = _u64(rsk)


class Server:
    def __init__(self, handle, prm: Params):
        self._h = handle
        self.prm = prm

    @classmethod
    def setup(cls, prm: Params, keys: PublicKeys, records, fmt: int = VIA_RECORDS_U64) -> "Server":
        """Server::setup: encode + prepare the database on the device, upload keys.

        records: for VIA_RECORDS_U64 an array of n_records*n_rec coefficients;
        for VIA_RECORDS_NIBBLE a uint8 array of n_records*n_rec/2 bytes.
        """
        L = _lib.lib()
        cp = prm.to_c()
        if len(keys.cascade_key) != prm.cascade_key_len or len(keys.conv_key) != prm.conv_key_len or \
                len(keys.rsk) != prm.rsk_len:
            raise BufferTooShort("public key buffers do not match the parameter set")
        k = _lib.ViaPublicKeys(_ptr(keys.cascade_key), _ptr(keys.conv_key), _ptr(keys.rsk))
        if fmt == VIA_RECORDS_U64:
            rec = _u64(records)
            n = rec.size // prm.n_rec
        else:
            rec = np.ascontiguousarray(records, dtype=np.uint8)
            n = rec.size * 2 // prm.n_rec
        h = ctypes.c_void_p()
        check(L.via_server_setup(ctypes.byref(cp), ctypes.byref(k), rec.ctypes.data_as(ctypes.c_void_p), n, fmt,
                                 ctypes.byref(h)))
        s = cls(h, prm)
        s._keys = keys
        return s

    def view(self, n_rec: int, keys: PublicKeys | None = None) -> "Server":
        """A handle over this server's prepared database (shared, not copied) that
        reads it as records of degree n_rec (via_server_view): VIA-C (n2) or a
        VIA-B n3. `keys` defaults to this server's keys."""
        keys = keys if keys is not None else self._keys
        prm = self.prm.with_dims(self.prm.num_rows, self.prm.num_cols, n_rec)
        k = _lib.ViaPublicKeys(_ptr(keys.cascade_key), _ptr(keys.conv_key), _ptr(keys.rsk))
        h = ctypes.c_void_p()
        check(_lib.lib().via_server_view(self._h, n_rec, ctypes.byref(k), ctypes.byref(h)))
        s = Server(h, prm)
        s._keys = keys
        return s

    def answer(self, query):
        """Server::answer: returns (mask mod q3, body mod q4), n2 residues each."""
        q = _u64(query)
        n_lwe = q.size // self.prm.lwe_len
        if n_lwe * self.prm.lwe_len != q.size:
            raise BufferTooShort("query buffer is not a whole number of LWEs")
        mask = np.zeros(self.prm.n2, dtype=np.uint64)
        body = np.zeros(self.prm.n2, dtype=np.uint64)
        check(_lib.lib().via_server_answer(self._h, _ptr(q), n_lwe, _ptr(mask), _ptr(body)))
        return mask, body

    def answer_many(self, queries):
        """Answers a batch of independent queries with one shared database pass.

        queries: (n, n_lwe * lwe_len) or flat; returns (masks, bodies), each (n, n2).
        """
        prm = self.prm
        q = _u64(queries).reshape(-1)
        per = prm.n_lwe * prm.lwe_len
        if q.size % per:
            raise BufferTooShort("query buffer is not a whole number of queries")
        n = q.size // per
        masks = np.zeros((n, prm.n2), dtype=np.uint64)
        bodies = np.zeros((n, prm.n2), dtype=np.uint64)
        check(_lib.lib().via_server_answer_many(self._h, _ptr(q), n, prm.n_lwe, _ptr(masks), _ptr(bodies)))
        return masks, bodies

    def reserve(self, max_queries: int) -> None:
        check(_lib.lib().via_server_reserve(self._h, max_queries))

    def debug_stage(self, query, stage: int) -> np.ndarray:
        """The answer's intermediate `stage` (1..7), see via_debug_stage in include/via_gpu.h."""
        prm = self.prm
        q = _u64(query)
        nbits = prm.n_lwe // prm.l_query
        size = {1: prm.n_lwe * 2 * prm.nl * prm.n1, 2: nbits * 2 * prm.l_query * 2 * prm.nl * prm.n1,
                3: prm.num_rows * 2 * prm.nl * prm.n1, 4: prm.num_rows * 2 * prm.n1, 5: prm.num_cols * 2 * prm.n1,
                6: 2 * prm.n1, 7: 2 * prm.n1}[stage]
        out = np.zeros(size, dtype=np.uint64)
        check(_lib.lib().via_debug_stage(self._h, _ptr(q), q.size // prm.lwe_len, stage, _ptr(out), size))
        return out

    def first_dim_dev(self, switched_ptr: int, out_ptr: int, stream: int = 0) -> None:
        """FirstDim on device buffers (I RLWEs at q2 in, J RLWEs out)."""
        check(_lib.lib().via_first_dim_dev(self._h, ctypes.c_void_p(switched_ptr), ctypes.c_void_p(out_ptr),
                                           ctypes.c_void_p(stream)))

    def answer_batch(self, queries):
        """Server::answer_batch (VIA-B): T = n2 / n_rec queries, one answer (mask, body).

        queries: (T, n_lwe * lwe_len). Raises DimMismatch when the count is not T and
        QueryLengthMismatch when a query does not hold n_lwe LWEs.
        """
        prm = self.prm
        q = np.ascontiguousarray(queries, dtype=np.uint64)
        if q.ndim != 2 or q.shape[1] % prm.lwe_len:
            raise BufferTooShort("queries must be (T, n_lwe * lwe_len)")
        mask = np.zeros(prm.n2, dtype=np.uint64)
        body = np.zeros(prm.n2, dtype=np.uint64)
        check(_lib.lib().via_server_answer_batch(self._h, q.ctypes.data_as(ctypes.c_void_p), q.shape[0],
                                                 q.shape[1] // prm.lwe_len, mask.ctypes.data_as(ctypes.c_void_p),
                                                 body.ctypes.data_as(ctypes.c_void_p)))
        return mask, body

    def scan_dev(self, sel_eval_ptr: int, out_eval_ptr: int, stream: int = 0) -> None:
        """The FirstDim scan alone on eval-form device buffers (one query)."""
        check(_lib.lib().via_first_dim_scan_dev(self._h, ctypes.c_void_p(sel_eval_ptr), ctypes.c_void_p(out_eval_ptr),
                                                ctypes.c_void_p(stream)))

    def transform_q2_dev(self, data_ptr: int, count: int, inverse: bool = False, stream: int = 0) -> None:
        """The server's own transform at (q2, n1), in place on `count` polynomials:
        the eval form scan_dev / scan_many_dev take and return."""
        check(_lib.lib().via_server_transform_q2_dev(self._h, ctypes.c_void_p(data_ptr), count, 1 if inverse else 0,
                                                     ctypes.c_void_p(stream)))

    def scan_many_dev(self, sel_eval_ptr: int, n_queries: int, out_eval_ptr: int, stream: int = 0) -> None:
        """The scans of n_queries queries in one pass over the database (eval form)."""
        check(_lib.lib().via_first_dim_scan_many_dev(self._h, ctypes.c_void_p(sel_eval_ptr), n_queries,
                                                     ctypes.c_void_p(out_eval_ptr), ctypes.c_void_p(stream)))

    def autotune(self, batch_sizes, cache_path: str | None = None) -> list:
        """Runs the scan autotuner for these batch sizes (via_server_autotune);
        returns one dict per size: the tile kept, its time and the default's."""
        sizes = (ctypes.c_uint32 * len(batch_sizes))(*[int(b) for b in batch_sizes])
        out = (_lib.ScanTuning * len(batch_sizes))()
        path = cache_path.encode() if cache_path else None
        check(_lib.lib().via_server_autotune(self._h, sizes, len(batch_sizes), path, out))
        return [o.as_dict() for o in out]

    def scan_tile_candidates(self, batch: int) -> list:
        """The tiles the autotuner tries for `batch` queries (default first)."""
        L = _lib.lib()
        n = int(L.via_scan_tile_candidates(self._h, batch, None, 0))
        out = (_lib.ScanTile * max(1, n))()
        L.via_scan_tile_candidates(self._h, batch, out, n)
        return [out[i].as_dict() for i in range(n)]

    def set_scan_tile(self, batch: int, tile: dict | None) -> None:
        """Forces (or, with None, clears) the scan tile for `batch` queries."""
        t = None
        if tile is not None:
            t = ctypes.byref(_lib.ScanTile(tile.get("n_max", 0), tile.get("stages", 0), tile.get("order", 0), 0))
        check(_lib.lib().via_server_set_scan_tile(self._h, batch, t))

    def set_scan_fault(self, wait_us: int) -> None:
        """Test hook (via_server_set_scan_fault): scans make a bounded wait run out
        after wait_us microseconds and report VIA_ERR_TIMEOUT; 0 turns it off."""
        check(_lib.lib().via_server_set_scan_fault(self._h, wait_us))

    def close(self) -> None:
        if self._h:
            _lib.lib().via_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
