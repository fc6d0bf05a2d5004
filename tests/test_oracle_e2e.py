"""End-to-end "recover == record" on the oracle (the reference's e2e property).

Mirrors crates/via-integration/tests/client_server_e2e.rs (n1=8 stack, seed
"via-c-client-server-e2e", all indices), client_server_e2e_paper.rs (paper
preset, I=J=2, index 15) and the TOY_PARAMS preset (never run end to end by the
reference; recovering here shows the preset is usable).
"""
import numpy as np
import pytest

from via_rs_b200.params import n8_preset, paper_preset, toy_preset
from via_rs_b200.prg import Shake256Prg, nibble_records, seed_bytes


def n8_records():
    # client_server_e2e.rs record(m)
    return np.array([[(m + 1) % 16, (2 * m + 1) % 16, (3 * m + 1) % 16, (m + 5) % 16] for m in range(8)],
                    dtype=np.uint64)


def paper_records(n, n2=512):
    # client_server_e2e_paper.rs record(m): first 4 coefficients (m+1+j) % 16.
    r = np.zeros((n, n2), dtype=np.uint64)
    for m in range(n):
        r[m, :4] = [(m + 1 + j) % 16 for j in range(4)]
    return r


def test_n8_all_indices(oracle):
    prm = n8_preset()
    recs = n8_records()
    client = oracle.Client(prm, b"via-c-client-server-e2e")
    server = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    prg_label = b"via-c-client-server-e2e-query"
    for idx in range(prm.capacity):
        q = client.query(idx, prg_label + bytes([idx]))
        mask, body = server.answer(q)
        assert (client.recover(mask, body) == recs[idx]).all(), idx


def test_toy_preset_recovers(oracle):
    prm = toy_preset()
    recs = nibble_records(Shake256Prg(seed_bytes(0)), prm.capacity, prm.n_rec)
    client = oracle.Client(prm, seed_bytes(1))
    server = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    prg = Shake256Prg(seed_bytes(2))
    for _ in range(3):
        idx = prg.uniform_below(prm.capacity)
        q = client.query(idx, seed_bytes(1000 + idx))
        mask, body = server.answer(q)
        assert (client.recover(mask, body) == recs[idx]).all(), idx


def test_paper_preset_2x2_index_15(oracle):
    prm = paper_preset(2, 2)
    recs = paper_records(prm.capacity)
    client = oracle.Client(prm, b"via-c-paper-scale-e2e")
    server = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    q = client.query(15, b"via-c-paper-scale-e2e-q")
    mask, body = server.answer(q)
    assert (client.recover(mask, body) == recs[15]).all()


def test_setup_errors_mirror_via_error(oracle):
    prm = n8_preset(num_rows=3)
    with pytest.raises(oracle.OracleError) as e:
        oracle.Client(prm, b"x")
    assert "powers of two" in str(e.value)


def test_query_length_mismatch(oracle):
    prm = n8_preset()
    client = oracle.Client(prm, b"qlm")
    server = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, n8_records())
    q = client.query(0, b"qlm-q")
    with pytest.raises(oracle.OracleError) as e:
        server.answer(q[: -prm.lwe_len])
    assert e.value.code == 3


def test_secure_preset_recovers(oracle):
    """SECURE_PARAMS (n1=4096, n2=1024, q4=2^15; client_server_e2e_secure.rs): recover == record."""
    from via_rs_b200.params import secure_preset

    prm = secure_preset(2, 2)
    rng = np.random.default_rng(4096)
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"via-c-secure-e2e")
    server = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    for idx in (3, prm.capacity - 1):
        mask, body = server.answer(client.query(idx, b"secure-q-%d" % idx))
        assert (client.recover(mask, body) == recs[idx]).all(), idx
