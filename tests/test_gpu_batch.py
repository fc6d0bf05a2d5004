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
