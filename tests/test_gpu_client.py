"""The device client (via_client_*) against the oracle's client: queries are
bit-exact for the same secret keys and PRG seeds, recovery equals the oracle's,
and GPU client -> GPU server -> GPU recover returns every record (VIA-C and
VIA-B)."""
import numpy as np
import pytest

from via_rs_b200.client import Client
from via_rs_b200.params import n8_preset, paper_preset, secure_preset, toy_preset
from via_rs_b200.server import IndexOutOfRange, PublicKeys, Server

pytestmark = pytest.mark.gpu

PRESETS = {
    "n8": lambda: n8_preset(),
    "toy": lambda: toy_preset(4, 4),
    "paper": lambda: paper_preset(4, 8),
    "paper_t8": lambda: paper_preset(2, 4, n_rec=64),
    "secure": lambda: secure_preset(2, 4),
}


def _clients(oracle, prm, seed):
    oc = oracle.Client(prm, seed)
    sk1, sk2 = oc.secret_keys()
    return oc, Client(prm, sk1, sk2)


@pytest.mark.parametrize("preset", sorted(PRESETS))
def test_queries_match_oracle(oracle, preset):
    prm = PRESETS[preset]()
    oc, gc = _clients(oracle, prm, b"client-" + preset.encode())
    rng = np.random.default_rng(len(preset))
    idx = [int(i) for i in rng.integers(prm.capacity, size=5)] + [0, prm.capacity - 1]
    seeds = [b"query-seed-%03d" % k for k in range(len(idx))]
    got = gc.queries(idx, seeds)
    for k, i in enumerate(idx):
        assert np.array_equal(got[k], oc.query(i, seeds[k])), f"{preset}: query {k} (index {i})"


def test_long_and_short_seeds(oracle):
    prm = paper_preset(2, 2)
    oc, gc = _clients(oracle, prm, b"client-seeds")
    for seed in (b"s", b"x" * 64):
        assert np.array_equal(gc.query(3, seed), oc.query(3, seed))


def test_recover_round_trip(oracle):
    prm = paper_preset(4, 8)
    rng = np.random.default_rng(9)
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    oc, gc = _clients(oracle, prm, b"client-rt")
    server = Server.setup(prm, PublicKeys(oc.cascade_key, oc.conv_key, oc.rsk), recs)
    idx = [int(i) for i in rng.integers(prm.capacity, size=12)]
    qs = gc.queries(idx, [b"rt-%02d" % k for k in range(len(idx))])
    masks, bodies = server.answer_many(qs)
    got = gc.recover_many(masks, bodies)
    for k, i in enumerate(idx):
        assert np.array_equal(got[k], recs[i]), (k, i)
        assert np.array_equal(got[k], oc.recover(masks[k], bodies[k]))


def test_via_b_round_trip(oracle):
    prm = paper_preset(2, 4, n_rec=64)
    rng = np.random.default_rng(10)
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    oc, gc = _clients(oracle, prm, b"client-b")
    server = Server.setup(prm, PublicKeys(oc.cascade_key, oc.conv_key, oc.rsk), recs)
    T = prm.n2 // prm.n_rec
    idx = [int(i) for i in rng.integers(prm.capacity, size=T)]
    qs = gc.queries(idx, [b"b-%02d" % k for k in range(T)])
    m, b = server.answer_batch(qs)
    for t, rec in enumerate(gc.recover_batch(m, b)):
        assert np.array_equal(rec, recs[idx[t]]), t


def test_index_out_of_range(oracle):
    prm = paper_preset(2, 2)
    _, gc = _clients(oracle, prm, b"client-oor")
    with pytest.raises(IndexOutOfRange):
        gc.queries([prm.capacity], [b"x"])
