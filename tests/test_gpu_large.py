"""The batched VIA-C workload at 4 GiB: 64 concurrent queries with seeded random
indices against a 4 GiB uniform random database (I = 2^9, J = 2^13, paper
preset), answered with one shared database scan. The oracle cannot hold this
database, so the checks are the size-independent properties: every answer
recovers its record, and the batched answers equal single-query answers."""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.server import VIA_RECORDS_NIBBLE, PublicKeys, Server

pytestmark = pytest.mark.gpu


def _nibbles(records_u8, i, n_rec):
    row = records_u8[i * n_rec // 2:(i + 1) * n_rec // 2]
    out = np.empty(n_rec, dtype=np.uint64)
    out[0::2] = row & 15
    out[1::2] = row >> 4
    return out


def test_batched_64_queries_4gib(oracle):
    prm = paper_preset(512, 8192)
    assert prm.capacity * prm.n_rec // 2 == 4 << 30
    rng = np.random.default_rng(4)
    records = rng.integers(0, 256, size=prm.capacity * prm.n_rec // 2, dtype=np.uint8)
    client = oracle.Client(prm, b"large-4gib")
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), records,
                       VIA_RECORDS_NIBBLE)
    idx = [int(i) for i in rng.integers(prm.capacity, size=64)]
    qs = np.stack([client.query(i, b"large-q%d" % k) for k, i in enumerate(idx)])
    masks, bodies = gpu.answer_many(qs)
    for k, i in enumerate(idx):
        assert np.array_equal(client.recover(masks[k], bodies[k]), _nibbles(records, i, prm.n_rec)), (k, i)
    for k in (0, 17, 63):
        m, b = gpu.answer(qs[k])
        assert np.array_equal(m, masks[k]) and np.array_equal(b, bodies[k]), f"query {k}: batched != single"
    gpu.close()
