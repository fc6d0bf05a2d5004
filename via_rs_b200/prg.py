"""The reference's seeded byte stream, for generating synthetic workloads.

`Shake256Prg` (crates/via-primitives/src/sampling/prg.rs:57-205): 136-byte
blocks, block i = SHAKE256(seed || le64(i)). Seeds for the benchmark configs are
"seed k" = the 8-byte little-endian encoding of k.
"""
import hashlib

import numpy as np

BLOCK = 136


def seed_bytes(k: int) -> bytes:
    return int(k).to_bytes(8, "little")


class Shake256Prg:
    def __init__(self, seed: bytes):
        if len(seed) > 64:
            raise ValueError("seed longer than 64 bytes")
        self.seed = bytes(seed)
        self.counter = 0
        self.buf = b""
        self.pos = 0

    def _refill(self) -> None:
        self.buf = hashlib.shake_256(self.seed + self.counter.to_bytes(8, "little")).digest(BLOCK)
        self.counter += 1
        self.pos = 0

    def bytes(self, n: int) -> bytes:
        out = bytearray()
        while len(out) < n:
            if self.pos >= len(self.buf):
                self._refill()
            take = min(n - len(out), len(self.buf) - self.pos)
            out += self.buf[self.pos:self.pos + take]
            self.pos += take
        return bytes(out)

    def uniform_below(self, bound: int) -> int:
        """prg.rs uniform_below: rejection sampling on the low bitlen(bound) bits."""
        if bound <= 0:
            raise ValueError("bound must be positive")
        if bound == 1:
            return 0
        bits = bound.bit_length()
        nbytes = (bits + 7) // 8
        mask = (1 << bits) - 1
        while True:
            v = int.from_bytes(self.bytes(nbytes), "little") & mask
            if v < bound:
                return v


def stream_bytes(seed: bytes, n: int) -> bytes:
    """The first n bytes of Shake256Prg(seed), computed block by block in one
    pass (the same bytes as Shake256Prg(seed).bytes(n), faster for large n)."""
    if len(seed) > 64:
        raise ValueError("seed longer than 64 bytes")
    blocks = (n + BLOCK - 1) // BLOCK
    h = hashlib.shake_256
    return b"".join([h(seed + i.to_bytes(8, "little")).digest(BLOCK) for i in range(blocks)])[:n]


def nibble_records(prg: Shake256Prg, n_records: int, n_rec: int) -> np.ndarray:
    """n_records records of n_rec 4-bit coefficients from the byte stream, two
    coefficients per byte, low nibble first. Returns uint64 coefficients."""
    raw = np.frombuffer(prg.bytes(n_records * n_rec // 2), dtype=np.uint8)
    out = np.empty(raw.size * 2, dtype=np.uint64)
    out[0::2] = raw & 15
    out[1::2] = raw >> 4
    return out.reshape(n_records, n_rec)
