"""Query wire packets (crates/via-protocol/src/wire/format.rs:93-190) and the
server calls that take them.

A wire query is one packet per LWE: Uncompressed (tag 0x00, the LWE verbatim)
or PrgCompressed (tag 0x01, a 32-byte seed and the body; the mask is
regenerated from Shake256Prg(seed) on the device).
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib
from .params import Params
from .server import Server, check

SEED_LEN = 32


def uncompressed_packet(lwe: np.ndarray) -> bytes:
    lwe = np.ascontiguousarray(lwe, dtype="<u8")
    return b"\x00" + struct.pack("<Q", lwe.size) + lwe.tobytes()


def prg_packet(seed: bytes, body: np.ndarray) -> bytes:
    if len(seed) != SEED_LEN:
        raise ValueError("PrgCompressed seeds are 32 bytes")
    body = np.ascontiguousarray(body, dtype="<u8")
    return b"\x01" + seed + struct.pack("<Q", body.size) + body.tobytes()


def encode_uncompressed(prm: Params, query: np.ndarray) -> bytes:
    q = np.ascontiguousarray(query, dtype=np.uint64).reshape(prm.n_lwe, prm.lwe_len)
    return b"".join(uncompressed_packet(l) for l in q)


def from_wire(server: Server, wire: bytes) -> np.ndarray:
    """The flat query a wire query decodes to (masks regenerated on the device)."""
    prm = server.prm
    out = np.zeros(prm.n_lwe * prm.lwe_len, dtype=np.uint64)
    buf = ctypes.create_string_buffer(wire, len(wire))
    check(_lib.lib().via_query_from_wire(server._h, buf, len(wire), out.ctypes.data_as(ctypes.c_void_p), out.size))
    return out


def answer_wire(server: Server, wire: bytes):
    prm = server.prm
    m = np.zeros(prm.n2, dtype=np.uint64)
    b = np.zeros(prm.n2, dtype=np.uint64)
    buf = ctypes.create_string_buffer(wire, len(wire))
    check(_lib.lib().via_server_answer_wire(server._h, buf, len(wire), m.ctypes.data_as(ctypes.c_void_p),
                                            b.ctypes.data_as(ctypes.c_void_p)))
    return m, b
