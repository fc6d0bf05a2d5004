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
