"""Plain VIA-C at paper scale on the full 1 GiB database, against the oracle.

The paper preset (n1 = 2048 over the two q1 primes, q2 = 17175674881) with
I = 2^8, J = 2^12: 2^22 records of 512 4-bit coefficients, the 1 GiB database
of the paper's Table 4. Records are the first 1 GiB of Shake256Prg("seed 0"),
the client's keys come from "seed 1" and the indices from "seed 2" ("seed k"
is the 8-byte little-endian k). The GPU answer must equal the oracle's answer
residue for residue, and the client must recover the record, as the
reference's paper-scale end-to-end test asserts
(crates/via-integration/tests/client_server_e2e_paper.rs:146-177).
"""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.prg import Shake256Prg, seed_bytes, stream_bytes
from via_rs_b200.server import VIA_RECORDS_NIBBLE, PublicKeys, Server

pytestmark = pytest.mark.gpu


def _record(packed: np.ndarray, idx: int, n_rec: int) -> np.ndarray:
    row = packed[idx * n_rec // 2:(idx + 1) * n_rec // 2]
    out = np.empty(n_rec, dtype=np.uint64)
    out[0::2] = row & 15
    out[1::2] = row >> 4
    return out


def test_paper_1gib_answer_bit_exact(oracle):
    prm = paper_preset(256, 4096)
    db_bytes = prm.capacity * prm.n_rec // 2
    assert db_bytes == 1 << 30
    packed = np.frombuffer(stream_bytes(seed_bytes(0), db_bytes), dtype=np.uint8)
    client = oracle.Client(prm, seed_bytes(1))
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), packed, VIA_RECORDS_NIBBLE)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, packed)
    prg = Shake256Prg(seed_bytes(2))
    # Two seeded indices plus the last record (row I-1, column J-1, slot d-1).
    indices = [prg.uniform_below(prm.capacity), prg.uniform_below(prm.capacity), prm.capacity - 1]
    for k, idx in enumerate(indices):
        q = client.query(idx, seed_bytes(2) + b"-%d" % k)
        gm, gb = gpu.answer(q)
        cm, cb = cpu.answer(q)
        bad = np.nonzero(np.concatenate([gm != cm, gb != cb]))[0]
        assert bad.size == 0, f"index {idx}: {bad.size} answer residues differ from the oracle, first at {bad[:8]}"
        assert np.array_equal(client.recover(gm, gb), _record(packed, idx, prm.n_rec)), f"index {idx}: recover != record"
    gpu.close()
