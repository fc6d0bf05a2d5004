"""VIA-B answer_batch on the GPU vs the oracle: bit-exact answers, every record recovered.

The batch shares one database scan over the T queries, then repacks the T CRot
outputs (the cascade-key suffix switched to q2) and runs RespComp once
(crates/via-server/src/batch.rs:72-163).
"""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.server import DimMismatch, PublicKeys, QueryLengthMismatch, Server

pytestmark = pytest.mark.gpu


def _setup(oracle, rows, cols, n3, seed):
    prm = paper_preset(rows, cols, n_rec=n3)
    rng = np.random.default_rng(len(seed))
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, seed)
    keys = PublicKeys(client.cascade_key, client.conv_key, client.rsk)
    return prm, recs, client, Server.setup(prm, keys, recs), oracle.Server(prm, client.cascade_key,
                                                                           client.conv_key, client.rsk, recs)


@pytest.mark.parametrize("rows,cols", [(2, 2), (4, 8)])
def test_answer_batch_t8_matches_oracle(oracle, rows, cols):
    prm, recs, client, gpu, cpu = _setup(oracle, rows, cols, 64, b"gpu-via-b-%d" % rows)
    rng = np.random.default_rng(rows)
    idx = [int(i) for i in rng.integers(prm.capacity, size=8)]
    qs = client.batch_query(idx, b"gpu-batch-q")
    gm, gb = gpu.answer_batch(qs)
    cm, cb = cpu.answer_batch(qs)
    assert np.array_equal(gm, cm), "batch answer mask differs from the oracle"
    assert np.array_equal(gb, cb), "batch answer body differs from the oracle"
    got = client.recover_batch(gm, gb)
    for t, i in enumerate(idx):
        assert np.array_equal(got[t], recs[i]), (t, i)


def test_answer_batch_rejects_wrong_sizes(oracle):
    prm, recs, client, gpu, _ = _setup(oracle, 2, 2, 64, b"gpu-via-b-err")
    qs = client.batch_query(list(range(8)), b"e")
    with pytest.raises(DimMismatch):
        gpu.answer_batch(qs[:4])
    with pytest.raises(QueryLengthMismatch):
        gpu.answer_batch(qs[:, : -prm.lwe_len])


@pytest.mark.parametrize("T", [2, 4, 16, 32, 64, 128, 256])
def test_answer_batch_every_t_matches_oracle(oracle, T):
    """Every power-of-two batch size T = n2 / n_rec, records of degree n2 / T (the
    reference's repack engine is generic over T, repack.rs:331-397; its record-fit
    rule admits any power of two with T * n_rec <= n2, presets.rs:170-176). The
    answer equals the oracle's and recover_batch returns every queried record.
    T = 256 (records of degree 2) is the production VIA-B batch: a depth-10 repack."""
    prm = paper_preset(2, 2, n_rec=512 // T)
    assert prm.n2 // prm.n_rec == T
    rng = np.random.default_rng(1000 + T)
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"gpu-via-b-t%d" % T)
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), recs)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    idx = [int(i) for i in rng.integers(prm.capacity, size=T)]
    qs = client.batch_query(idx, b"t%d" % T)
    gm, gb = gpu.answer_batch(qs)
    cm, cb = cpu.answer_batch(qs)
    assert np.array_equal(gm, cm), f"T={T}: batch answer mask differs from the oracle"
    assert np.array_equal(gb, cb), f"T={T}: batch answer body differs from the oracle"
    got = client.recover_batch(gm, gb)
    bad = [t for t, i in enumerate(idx) if not np.array_equal(got[t], recs[i])]
    assert not bad, f"T={T}: {len(bad)} records wrong, first slots {bad[:8]}"
    gpu.close()
