"""ctypes binding of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as
the checker. The product path (via_rs_b200) never imports this module.
"""
import ctypes
import os
import pathlib

import numpy as np

from via_rs_b200.params import Params

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "_build" / "libvia_oracle.so"

_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (g++)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.vo_last_error.restype = ctypes.c_char_p
        L.vo_kat.restype = ctypes.c_long
        L.vo_kat.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _u64p, ctypes.c_size_t]
        L.vo_client_setup.restype = ctypes.c_void_p
        L.vo_client_setup.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, _u64p, _u64p, _u64p]
        L.vo_client_query.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_char_p,
                                      ctypes.c_size_t, _u64p]
        L.vo_client_recover.argtypes = [ctypes.c_void_p, _u64p, _u64p, _u64p]
        L.vo_client_free.argtypes = [ctypes.c_void_p]
        L.vo_client_secret.argtypes = [ctypes.c_void_p, _u64p, _u64p]
        L.vo_server_setup.restype = ctypes.c_void_p
        L.vo_server_setup.argtypes = [ctypes.c_void_p, _u64p, _u64p, _u64p, _u64p, ctypes.c_size_t, ctypes.c_int]
        L.vo_server_setup_packed.restype = ctypes.c_void_p
        L.vo_server_setup_packed.argtypes = [ctypes.c_void_p, _u64p, _u64p, _u64p, ctypes.c_void_p, ctypes.c_size_t,
                                             ctypes.c_int]
        L.vo_server_answer.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, _u64p, _u64p, ctypes.c_int]
        L.vo_server_answer_batch.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p, _u64p,
                                             ctypes.c_int]
        L.vo_server_answer_through_crot.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, _u64p, ctypes.c_int]
        L.vo_server_first_dim.argtypes = [ctypes.c_void_p, _u64p, _u64p, ctypes.c_int]
        L.vo_server_free.argtypes = [ctypes.c_void_p]
        L.vo_server_debug_stage.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t, ctypes.c_int, _u64p, ctypes.c_int]
        L.vo_stage_times.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.vo_shake256.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
        L.vo_gadget_digits.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _u64p,
                                       ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64)]
        L.vo_ntt.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _u64p, ctypes.c_size_t]
        L.vo_external_product.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64,
                                          ctypes.c_int, _u64p, _u64p, ctypes.c_size_t, _u64p, ctypes.c_int]
        L.vo_key_switch.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                    _u64p, _u64p, _u64p, ctypes.c_size_t, _u64p, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def stage_len(prm: Params, stage: int) -> int:
    nl, n1 = prm.nl, prm.n1
    nbits = prm.n_lwe // prm.l_query
    return {1: prm.n_lwe * 2 * nl * n1, 2: nbits * 2 * prm.l_query * 2 * nl * n1, 3: prm.num_rows * 2 * nl * n1,
            4: prm.num_rows * 2 * n1, 5: prm.num_cols * 2 * n1, 6: 2 * n1, 7: 2 * n1}[stage]


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(rc, lib().vo_last_error().decode())


def shake256(data: bytes, n: int) -> bytes:
    out = ctypes.create_string_buffer(n)
    lib().vo_shake256(data, len(data), out, n)
    return out.raw


def kat(layer: str, scenario: str, name: str, cap: int = 4096) -> np.ndarray:
    out = np.zeros(cap, dtype=np.uint64)
    n = lib().vo_kat(layer.encode(), scenario.encode(), name.encode(), _ptr(out), cap)
    if n < 0:
        raise OracleError(-n, f"{layer}/{scenario}/{name}: " + lib().vo_last_error().decode())
    return out[:n].copy()


def _u64c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def gadget_digits(q: tuple, base: int, L: int, coeffs) -> np.ndarray:
    """Balanced gadget digits (gadget.rs:115-190) of coefficients [count][nl]: [count][L]."""
    c = _u64c(coeffs)
    count = c.size // len(q)
    out = np.zeros(count * L, dtype=np.int64)
    q1 = q[1] if len(q) > 1 else 0
    _check(lib().vo_gadget_digits(q[0], q1, base, L, _ptr(c), count, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
    return out.reshape(count, L)


def ntt(q: tuple, n: int, data, inverse: bool = False) -> np.ndarray:
    """The reference's negacyclic NTT (ntt.rs:305-399) of [count][nl][n] residues
    over the primes q = (q0,) or (q0, q1); returns a new array."""
    out = _u64c(data).copy()
    q1 = q[1] if len(q) > 1 else 0
    _check(lib().vo_ntt(q[0], q1, n, 1 if inverse else 0, _ptr(out), out.size // (len(q) * n)))
    return out


def external_product(q: tuple, n: int, base: int, L: int, rgsw, rlwe, threads: int = 0) -> np.ndarray:
    """RGSW (x) RLWE (rgsw.rs:108-121) per pair: rgsw [c][2L][2][nl][n], rlwe [c][2][nl][n]."""
    rg, ct = _u64c(rgsw), _u64c(rlwe)
    nl = len(q)
    count = ct.size // (2 * nl * n)
    out = np.zeros(count * 2 * nl * n, dtype=np.uint64)
    q1 = q[1] if nl > 1 else 0
    _check(lib().vo_external_product(q[0], q1, n, base, L, _ptr(rg), _ptr(ct), count, _ptr(out),
                                     threads or os.cpu_count() or 1))
    return out


def key_switch(q: tuple, n: int, base: int, L: int, key, rlwe, shifts, threads: int = 0) -> np.ndarray:
    """key_switch(key, X^k ct) (keyswitch.rs:99-102, element.rs:328) per ciphertext."""
    k, ct, sh = _u64c(key), _u64c(rlwe), _u64c(shifts)
    nl = len(q)
    count = ct.size // (2 * nl * n)
    out = np.zeros(count * 2 * nl * n, dtype=np.uint64)
    q1 = q[1] if nl > 1 else 0
    _check(lib().vo_key_switch(q[0], q1, n, base, L, _ptr(k), _ptr(ct), _ptr(sh), count, _ptr(out),
                               threads or os.cpu_count() or 1))
    return out


class Client:
    """Client::setup / query / recover (crates/via-client/src/client.rs)."""

    def __init__(self, prm: Params, seed: bytes):
        self.prm = prm
        self.cascade_key = np.zeros(prm.cascade_key_len, dtype=np.uint64)
        self.conv_key = np.zeros(prm.conv_key_len, dtype=np.uint64)
        self.rsk = np.zeros(prm.rsk_len, dtype=np.uint64)
        self._cp = prm.to_c()
        h = lib().vo_client_setup(ctypes.byref(self._cp), seed, len(seed), _ptr(self.cascade_key),
                                  _ptr(self.conv_key), _ptr(self.rsk))
        if not h:
            raise OracleError(-1, lib().vo_last_error().decode())
        self._h = h

    def query(self, index: int, seed: bytes, d: int | None = None) -> np.ndarray:
        prm = self.prm
        d = prm.n1 // prm.n_rec if d is None else d
        n = (prm.num_dmux + prm.num_cmux + (d.bit_length() - 1 if d > 1 else 0)) * prm.l_query
        out = np.zeros(n * prm.lwe_len, dtype=np.uint64)
        _check(lib().vo_client_query(self._h, index, d, seed, len(seed), _ptr(out)))
        return out

    def batch_query(self, indices, seed: bytes) -> np.ndarray:
        """Client::batch_query (cli/client.rs:256-300): one query per index at d3 = n1 / n_rec."""
        return np.stack([self.query(int(i), seed + b"-%d" % k) for k, i in enumerate(indices)])

    def secret_keys(self):
        """(S1 [nl * n1] at q1, S2 [n2] at q3), for the device client's tests."""
        prm = self.prm
        sk1 = np.zeros(prm.nl * prm.n1, dtype=np.uint64)
        sk2 = np.zeros(prm.n2, dtype=np.uint64)
        lib().vo_client_secret(self._h, _ptr(sk1), _ptr(sk2))
        return sk1, sk2

    def recover_batch(self, mask: np.ndarray, body: np.ndarray) -> list:
        """Client::recover_batch (cli/client.rs:316-333, cli/batch.rs:35-58): record t is
        project_at::<n_rec>(t) of the recovered degree-n2 plaintext."""
        plain = self.recover(mask, body)
        stride = self.prm.n2 // self.prm.n_rec
        return [plain[t::stride] for t in range(stride)]

    def recover(self, mask: np.ndarray, body: np.ndarray) -> np.ndarray:
        out = np.zeros(self.prm.n2, dtype=np.uint64)
        _check(lib().vo_client_recover(self._h, _ptr(np.ascontiguousarray(mask, dtype=np.uint64)),
                                       _ptr(np.ascontiguousarray(body, dtype=np.uint64)), _ptr(out)))
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib().vo_client_free(self._h)
            self._h = None


class Server:
    """Server::setup / answer on the CPU (crates/via-server/src/answer.rs)."""

    def __init__(self, prm: Params, cascade_key, conv_key, rsk, records: np.ndarray, threads: int = 0):
        """records: u64 coefficients [n_records][n_rec], or a uint8 array of 4-bit
        coefficients packed two per byte, low nibble first (n_records * n_rec / 2 bytes)."""
        self.prm = prm
        self.threads = threads or os.cpu_count() or 1
        self._cp = prm.to_c()
        if records.dtype == np.uint8:
            rec = np.ascontiguousarray(records).reshape(-1)
            n_rec = rec.size * 2 // prm.n_rec
            h = lib().vo_server_setup_packed(ctypes.byref(self._cp), _ptr(cascade_key), _ptr(conv_key), _ptr(rsk),
                                             rec.ctypes.data_as(ctypes.c_void_p), n_rec, self.threads)
        else:
            rec = np.ascontiguousarray(records, dtype=np.uint64)
            n_rec = rec.size // prm.n_rec
            h = lib().vo_server_setup(ctypes.byref(self._cp), _ptr(cascade_key), _ptr(conv_key), _ptr(rsk),
                                      _ptr(rec), n_rec, self.threads)
        if not h:
            raise OracleError(-1, lib().vo_last_error().decode())
        self._h = h

    def answer(self, query: np.ndarray):
        prm = self.prm
        q = np.ascontiguousarray(query, dtype=np.uint64)
        mask = np.zeros(prm.n2, dtype=np.uint64)
        body = np.zeros(prm.n2, dtype=np.uint64)
        _check(lib().vo_server_answer(self._h, _ptr(q), q.size // prm.lwe_len, _ptr(mask), _ptr(body),
                                      self.threads))
        return mask, body

    def answer_batch(self, queries: np.ndarray):
        """Server::answer_batch (srv/batch.rs:72-163): queries (T, n_lwe * lwe_len), one answer."""
        prm = self.prm
        q = np.ascontiguousarray(queries, dtype=np.uint64)
        if q.ndim != 2:
            raise ValueError("queries must be (T, n_lwe * lwe_len)")
        mask = np.zeros(prm.n2, dtype=np.uint64)
        body = np.zeros(prm.n2, dtype=np.uint64)
        _check(lib().vo_server_answer_batch(self._h, _ptr(q), q.shape[0], q.shape[1] // prm.lwe_len, _ptr(mask),
                                            _ptr(body), self.threads))
        return mask, body

    def answer_through_crot(self, query: np.ndarray) -> np.ndarray:
        prm = self.prm
        q = np.ascontiguousarray(query, dtype=np.uint64)
        out = np.zeros(2 * prm.n1, dtype=np.uint64)
        _check(lib().vo_server_answer_through_crot(self._h, _ptr(q), q.size // prm.lwe_len, _ptr(out),
                                                   self.threads))
        return out

    def first_dim(self, switched: np.ndarray) -> np.ndarray:
        prm = self.prm
        out = np.zeros(prm.num_cols * 2 * prm.n1, dtype=np.uint64)
        _check(lib().vo_server_first_dim(self._h, _ptr(np.ascontiguousarray(switched, dtype=np.uint64)),
                                         _ptr(out), self.threads))
        return out

    def debug_stage(self, query: np.ndarray, stage: int) -> np.ndarray:
        """Intermediate `stage` (1..7) in the layout of include/via_gpu.h via_debug_stage."""
        prm = self.prm
        q = np.ascontiguousarray(query, dtype=np.uint64)
        out = np.zeros(stage_len(prm, stage), dtype=np.uint64)
        _check(lib().vo_server_debug_stage(self._h, _ptr(q), q.size // prm.lwe_len, stage, _ptr(out), self.threads))
        return out

    @staticmethod
    def stage_times():
        t = (ctypes.c_double * 7)()
        lib().vo_stage_times(t)
        return list(t)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().vo_server_free(self._h)
            self._h = None
