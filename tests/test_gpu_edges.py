"""Edge cases of Server::setup / answer on the device: capacity and shape errors
(the reference's ViaError::DimMismatch), a database with fewer records than
capacity (zero padding), a server without keys (SetupNotComplete), and the
largest number of rows the tensor-core scan takes (4096) against the first
one it refuses."""
import ctypes

import numpy as np
import pytest

from via_rs_b200 import _lib
from via_rs_b200.params import paper_preset
from via_rs_b200.server import VIA_RECORDS_NIBBLE, DimMismatch, PublicKeys, Server, SetupNotComplete, ViaError

pytestmark = pytest.mark.gpu


def _keys(oracle, prm, seed):
    c = oracle.Client(prm, seed)
    return c, PublicKeys(c.cascade_key, c.conv_key, c.rsk)


def _nibbles(records_u8, i, n_rec):
    row = records_u8[i * n_rec // 2:(i + 1) * n_rec // 2]
    out = np.empty(n_rec, dtype=np.uint64)
    out[0::2] = row & 15
    out[1::2] = row >> 4
    return out


def test_more_records_than_capacity(oracle):
    prm = paper_preset(2, 2)
    _, keys = _keys(oracle, prm, b"edge-cap")
    recs = np.zeros((prm.capacity + 1, prm.n_rec), dtype=np.uint64)
    with pytest.raises(DimMismatch):
        Server.setup(prm, keys, recs)


def test_non_power_of_two_grid(oracle):
    prm = paper_preset(2, 2)
    _, keys = _keys(oracle, prm, b"edge-pow2")
    bad = prm.with_dims(3, 2)
    with pytest.raises(DimMismatch):
        Server.setup(bad, keys, np.zeros((1, bad.n_rec), dtype=np.uint64))


def test_fewer_records_are_zero_padded(oracle):
    prm = paper_preset(2, 4)
    client, keys = _keys(oracle, prm, b"edge-pad")
    rng = np.random.default_rng(3)
    n = prm.capacity // 2 + 3
    recs = rng.integers(0, 16, size=(n, prm.n_rec), dtype=np.uint64)
    gpu = Server.setup(prm, keys, recs)
    for idx in (0, n - 1, n, prm.capacity - 1):
        m, b = gpu.answer(client.query(idx, b"pad-%d" % idx))
        want = recs[idx] if idx < n else np.zeros(prm.n_rec, dtype=np.uint64)
        assert np.array_equal(client.recover(m, b), want), idx


def test_answer_without_keys_is_setup_not_complete(oracle):
    prm = paper_preset(2, 2)
    client, _ = _keys(oracle, prm, b"edge-nokeys")
    L = _lib.lib()
    cp = prm.to_c()
    recs = np.zeros((prm.capacity, prm.n_rec), dtype=np.uint64)
    h = ctypes.c_void_p()
    rc = L.via_server_setup(ctypes.byref(cp), None, recs.ctypes.data_as(ctypes.c_void_p), prm.capacity, 0,
                            ctypes.byref(h))
    assert rc == 0, L.via_last_error()
    srv = Server(h, prm)
    with pytest.raises(SetupNotComplete):
        srv.answer(client.query(0, b"nokeys"))
    srv.close()


def test_largest_row_count(oracle):
    """4096 rows, the most the byte-plane scan's 32-bit accumulators allow."""
    prm = paper_preset(4096, 2)
    client, keys = _keys(oracle, prm, b"edge-rows")
    rng = np.random.default_rng(4)
    recs = rng.integers(0, 256, size=prm.capacity * prm.n_rec // 2, dtype=np.uint8)
    gpu = Server.setup(prm, keys, recs, VIA_RECORDS_NIBBLE)
    for idx in (0, prm.capacity - 1, int(rng.integers(prm.capacity))):
        m, b = gpu.answer(client.query(idx, b"rows-%d" % idx))
        assert np.array_equal(client.recover(m, b), _nibbles(recs, idx, prm.n_rec)), idx
    gpu.close()
    too_many = paper_preset(8192, 2)
    _, keys2 = _keys(oracle, too_many, b"edge-rows2")
    with pytest.raises(ViaError):
        Server.setup(too_many, keys2, np.zeros((1, too_many.n_rec), dtype=np.uint64))
