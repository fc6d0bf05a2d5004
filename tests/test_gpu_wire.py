"""Wire-format ingest on the GPU: PrgCompressed masks equal Shake256Prg's draws,
Uncompressed packets round-trip, and a wire query answers like the flat one."""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.prg import Shake256Prg
from via_rs_b200.server import BufferTooShort, PublicKeys, Server, UnknownFormatTag
from via_rs_b200.wire import answer_wire, encode_uncompressed, from_wire, prg_packet, uncompressed_packet

pytestmark = pytest.mark.gpu


def regenerate_mask(prm, seed):
    """format.rs:146-160: uniform_below(q_l) row-major, one draw per limb, limb 0 first."""
    prg = Shake256Prg(seed)
    nl = len(prm.q1)
    mask = np.zeros((nl, prm.n1), dtype=np.uint64)
    for k in range(prm.n1):
        for l in range(nl):
            mask[l, k] = prg.uniform_below(prm.q1[l])
    return mask.reshape(-1)


@pytest.fixture(scope="module")
def setup(oracle):
    prm = paper_preset(2, 4)
    rng = np.random.default_rng(21)
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"wire")
    return prm, recs, client, Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), recs)


def test_prg_compressed_masks_match_shake256prg(setup):
    prm, _, _, gpu = setup
    rng = np.random.default_rng(5)
    packets, want = [], []
    for w in range(prm.n_lwe):
        body = rng.integers(0, min(prm.q1), size=len(prm.q1), dtype=np.uint64)
        if w % 3 == 2:  # mixed packets: every third LWE verbatim
            lwe = np.concatenate([rng.integers(0, min(prm.q1), size=len(prm.q1) * prm.n1, dtype=np.uint64), body])
            packets.append(uncompressed_packet(lwe))
            want.append(lwe)
        else:
            seed = bytes(rng.integers(0, 256, size=32, dtype=np.uint8))
            packets.append(prg_packet(seed, body))
            want.append(np.concatenate([regenerate_mask(prm, seed), body]))
    got = from_wire(gpu, b"".join(packets))
    assert np.array_equal(got, np.concatenate(want))


def test_wire_answer_equals_flat_answer(setup):
    prm, recs, client, gpu = setup
    q = client.query(5, b"wire-q")
    assert np.array_equal(from_wire(gpu, encode_uncompressed(prm, q)), q)
    wm, wb = answer_wire(gpu, encode_uncompressed(prm, q))
    fm, fb = gpu.answer(q)
    assert np.array_equal(wm, fm) and np.array_equal(wb, fb)
    assert np.array_equal(client.recover(wm, wb), recs[5])


def test_wire_errors(setup):
    prm, _, client, gpu = setup
    wire = encode_uncompressed(prm, client.query(1, b"e"))
    with pytest.raises(UnknownFormatTag):
        from_wire(gpu, b"\x07" + wire[1:])
    with pytest.raises(BufferTooShort):
        from_wire(gpu, wire[: len(wire) // 2])
