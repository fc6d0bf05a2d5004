"""The answer path at NTT-friendly q2 primes above the presets' 2^34.

Every preset's q2 is below 2^34, where the byte-plane database stores the top
byte of each residue at two bits; these moduli take the five-plane layout of the
tensor-core scan instead, the double-precision q2 transforms with phase-boundary
reductions (35 bits) and the 64-bit integer ones (38 bits). Exact equality with
the oracle, plus recovery of the queried record.
"""
import dataclasses

import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.server import PublicKeys, Server

pytestmark = pytest.mark.gpu

# Primes q = 1 (mod 8192) just below 2^35 and 2^38.
Q2_WIDE = [34_359_697_409, 274_877_816_833]


def _setup(oracle, prm, records, seed):
    client = oracle.Client(prm, seed)
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), records)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, records)
    return client, gpu, cpu


@pytest.mark.parametrize("q2", Q2_WIDE)
def test_first_dim_wide_q2(oracle, q2):
    """Random and all-(q2-1) selections over two row chunks and two column tiles."""
    import torch

    prm = dataclasses.replace(paper_preset(128, 256), q2=q2)
    rng = np.random.default_rng(q2 % 997)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    records[: prm.capacity // 4] = 15
    client, gpu, cpu = _setup(oracle, prm, records, b"wide-fd-%d" % q2)
    for sel in (rng.integers(0, q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64),
                np.full(prm.num_rows * 2 * prm.n1, q2 - 1, dtype=np.uint64)):
        want = cpu.first_dim(sel)
        d_in = torch.from_numpy(sel.view(np.int64)).cuda()
        d_out = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
        gpu.first_dim_dev(d_in.data_ptr(), d_out.data_ptr())
        assert np.array_equal(d_out.cpu().numpy().view(np.uint64), want)


@pytest.mark.parametrize("q2", Q2_WIDE)
def test_answers_wide_q2(oracle, q2):
    """Single answers and one shared-scan batch equal the oracle's answers."""
    prm = dataclasses.replace(paper_preset(8, 16), q2=q2)
    rng = np.random.default_rng(q2 % 991)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"wide-ans-%d" % q2)
    idx = [0, prm.capacity - 1, int(rng.integers(prm.capacity))]
    qs = np.stack([client.query(i, b"wq-%d" % k) for k, i in enumerate(idx)])
    gm, gb = gpu.answer_many(qs)
    for k, i in enumerate(idx):
        cm, cb = cpu.answer(qs[k])
        sm, sb = gpu.answer(qs[k])
        assert np.array_equal(sm, cm) and np.array_equal(sb, cb), k
        assert np.array_equal(gm[k], cm) and np.array_equal(gb[k], cb), k
        assert np.array_equal(client.recover(cm, cb), records[i])
