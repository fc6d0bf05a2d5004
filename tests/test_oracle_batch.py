"""VIA-B on the oracle: answer_batch + recover_batch return every record.

Mirrors crates/via-integration/tests/batch_e2e_paper.rs: paper rings and moduli,
T = 8 records of degree n3 = 64 (T * n3 = n2), I = J = 2, the repack keys
derived from the RNS-q1 cascade key by the q1 -> q2 switch, and the reference's
record(m) = ((m + 1) * (j + 1)) % 16 and indices.
"""
import numpy as np

from via_rs_b200.params import paper_preset


def batch_records(n, n3):
    j = np.arange(n3, dtype=np.uint64) + 1
    return np.stack([((m + 1) * j) % 16 for m in range(n)]).astype(np.uint64)


def test_paper_batch_t8_recovers_every_record(oracle):
    prm = paper_preset(2, 2, n_rec=64)
    assert prm.n2 // prm.n_rec == 8
    recs = batch_records(prm.capacity, prm.n_rec)
    client = oracle.Client(prm, b"via-b-paper-batch-e2e")
    server = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    idx = [3, 17, 42, 5, 88, 100, 7, 120]
    mask, body = server.answer_batch(client.batch_query(idx, b"via-b-batch-query"))
    got = client.recover_batch(mask, body)
    assert len(got) == 8
    for t, i in enumerate(idx):
        assert np.array_equal(got[t], recs[i]), f"slot {t} must recover record {i}"


def test_batch_other_t_recovers_and_threading_is_exact(oracle):
    """T = 4 (records of degree 128): the generic repack recovers every record,
    and the checker's threaded prefixes give the single-threaded answer."""
    prm = paper_preset(2, 2, n_rec=128)
    assert prm.n2 // prm.n_rec == 4
    recs = batch_records(prm.capacity, prm.n_rec)
    client = oracle.Client(prm, b"via-b-t4")
    idx = [1, 30, 7, 12]
    qs = client.batch_query(idx, b"via-b-t4-q")
    one = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs, threads=1)
    many = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs, threads=4)
    m1, b1 = one.answer_batch(qs)
    m4, b4 = many.answer_batch(qs)
    assert np.array_equal(m1, m4) and np.array_equal(b1, b4)
    got = client.recover_batch(m4, b4)
    for t, i in enumerate(idx):
        assert np.array_equal(got[t], recs[i]), f"slot {t} must recover record {i}"


def test_packed_records_setup_equals_u64_setup(oracle):
    """The oracle's 4-bit packed record input (two coefficients per byte, low
    nibble first) prepares the same database as the u64 input."""
    prm = paper_preset(2, 4)
    rng = np.random.default_rng(3)
    packed = rng.integers(0, 256, size=prm.capacity * prm.n_rec // 2, dtype=np.uint8)
    recs = np.empty(packed.size * 2, dtype=np.uint64)
    recs[0::2] = packed & 15
    recs[1::2] = packed >> 4
    client = oracle.Client(prm, b"packed")
    a = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs.reshape(prm.capacity, prm.n_rec))
    b = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, packed)
    sel = rng.integers(0, prm.q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64)
    assert np.array_equal(a.first_dim(sel), b.first_dim(sel))
