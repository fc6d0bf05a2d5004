"""CUDA answer path vs the CPU oracle: bit-exact, through the C ABI.

All integer work, so the bar is exact equality of every residue, plus the
reference's end-to-end property (the client recovers the queried record).
"""
import numpy as np
import pytest

from via_rs_b200.params import n8_preset, paper_preset, secure_preset, toy_preset
from via_rs_b200.prg import Shake256Prg, nibble_records, seed_bytes
from via_rs_b200.server import PublicKeys, QueryLengthMismatch, Server

pytestmark = pytest.mark.gpu


def _setup(oracle, prm, records, seed):
    client = oracle.Client(prm, seed)
    keys = PublicKeys(client.cascade_key, client.conv_key, client.rsk)
    gpu = Server.setup(prm, keys, records)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, records)
    return client, gpu, cpu


def _check_answer(client, gpu, cpu, records, idx, qseed):
    q = client.query(idx, qseed)
    gm, gb = gpu.answer(q)
    cm, cb = cpu.answer(q)
    assert np.array_equal(gm, cm), "answer mask differs from the oracle"
    assert np.array_equal(gb, cb), "answer body differs from the oracle"
    assert np.array_equal(client.recover(gm, gb), records[idx]), "recover != record"


@pytest.mark.parametrize("preset", ["n8", "toy", "paper"])
@pytest.mark.parametrize("stage", [1, 2, 3, 4, 5, 6, 7])
def test_stage_parity(oracle, preset, stage):
    """Every intermediate of the answer (cascade RLWEs, query RGSWs, DMux outputs,
    switched rows, FirstDim columns, CMux and CRot outputs) equals the oracle's."""
    prm = {"n8": n8_preset(), "toy": toy_preset(4, 4), "paper": paper_preset(4, 4)}[preset]
    rng = np.random.default_rng(stage)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"stage-%s" % preset.encode())
    q = client.query(int(rng.integers(prm.capacity)), b"stage-q")
    got = gpu.debug_stage(q, stage)
    want = cpu.debug_stage(q, stage)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"stage {stage}: {bad.size} residues differ, first at {bad[:8]}"


def test_first_dim_matches_oracle(oracle):
    import torch

    prm = paper_preset(16, 32)
    rng = np.random.default_rng(11)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"fd-parity")
    sel = rng.integers(0, prm.q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64)
    want = cpu.first_dim(sel)
    d_in = torch.from_numpy(sel.view(np.int64)).cuda()
    d_out = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    gpu.first_dim_dev(d_in.data_ptr(), d_out.data_ptr())
    got = d_out.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, want)


def test_first_dim_edge_values(oracle):
    """All-(q2-1) selection and all-15 database: the largest exact sums."""
    import torch

    prm = paper_preset(64, 8)
    records = np.full((prm.capacity, prm.n_rec), 15, dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"fd-edge")
    sel = np.full(prm.num_rows * 2 * prm.n1, prm.q2 - 1, dtype=np.uint64)
    want = cpu.first_dim(sel)
    d_in = torch.from_numpy(sel.view(np.int64)).cuda()
    d_out = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    gpu.first_dim_dev(d_in.data_ptr(), d_out.data_ptr())
    assert np.array_equal(d_out.cpu().numpy().view(np.uint64), want)


def test_answer_n8_all_indices(oracle):
    prm = n8_preset()
    records = np.array([[(m + 1) % 16, (2 * m + 1) % 16, (3 * m + 1) % 16, (m + 5) % 16] for m in range(8)],
                       dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"via-c-client-server-e2e")
    for idx in range(prm.capacity):
        _check_answer(client, gpu, cpu, records, idx, b"n8-q" + bytes([idx]))


def test_answer_toy_preset(oracle):
    """Config 1: TOY_PARAMS, 1024 records from seed 0, keys seed 1, index seed 2."""
    prm = toy_preset()
    records = nibble_records(Shake256Prg(seed_bytes(0)), prm.capacity, prm.n_rec)
    client, gpu, cpu = _setup(oracle, prm, records, seed_bytes(1))
    prg = Shake256Prg(seed_bytes(2))
    for _ in range(4):
        idx = prg.uniform_below(prm.capacity)
        _check_answer(client, gpu, cpu, records, idx, seed_bytes(2) + bytes([idx % 256]))


@pytest.mark.parametrize("rows,cols", [(2, 2), (4, 8), (32, 16)])
def test_answer_paper_preset(oracle, rows, cols):
    prm = paper_preset(rows, cols)
    rng = np.random.default_rng(rows * 1000 + cols)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"paper-%d-%d" % (rows, cols))
    for idx in (0, prm.capacity - 1, int(rng.integers(prm.capacity))):
        _check_answer(client, gpu, cpu, records, idx, b"pq-%d" % idx)


def test_answer_rejects_wrong_query_length(oracle):
    prm = n8_preset()
    records = np.zeros((prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, _ = _setup(oracle, prm, records, b"qlm")
    q = client.query(0, b"qlm-q")
    with pytest.raises(QueryLengthMismatch):
        gpu.answer(q[: -prm.lwe_len])


@pytest.mark.parametrize("preset", ["n8", "toy", "paper"])
def test_answer_many_equals_single_answers(oracle, preset):
    """A batch shares one database pass; every answer equals the oracle's single answer."""
    prm = {"n8": n8_preset(), "toy": toy_preset(4, 8), "paper": paper_preset(8, 16)}[preset]
    rng = np.random.default_rng(99)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"many-%s" % preset.encode())
    for nq in (1, 3, 9):  # exercises the 8-, 4- and 1-query scan kernels
        idx = [int(i) for i in rng.integers(prm.capacity, size=nq)]
        qs = np.stack([client.query(i, b"mq-%d-%d" % (nq, k)) for k, i in enumerate(idx)])
        gm, gb = gpu.answer_many(qs)
        for k, i in enumerate(idx):
            cm, cb = cpu.answer(qs[k])
            assert np.array_equal(gm[k], cm) and np.array_equal(gb[k], cb), (nq, k)
            assert np.array_equal(client.recover(gm[k], gb[k]), records[i])


def _scan_setup(oracle, rows, cols, seed):
    prm = paper_preset(rows, cols)
    rng = np.random.default_rng(seed)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"scan-%d" % seed)
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), records)
    return prm, rng, gpu


@pytest.mark.parametrize("nq", [2, 9, 24, 25, 64])
def test_scan_many_equals_single_scans(oracle, nq):
    """The shared scan of nq queries (grouped tensor-core tiles, several column
    tiles and row chunks) equals nq single-query scans, which are pinned to the
    oracle above."""
    import torch

    prm, rng, gpu = _scan_setup(oracle, 128, 256, 5)
    sel = rng.integers(0, prm.q2, size=(nq, prm.num_rows * 2 * prm.n1), dtype=np.uint64)
    if nq == 25:
        sel[3] = prm.q2 - 1  # largest exact sums in one column of the batch
    d_sel = torch.from_numpy(sel.view(np.int64)).cuda()
    d_many = torch.empty(nq * prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    gpu.scan_many_dev(d_sel.data_ptr(), nq, d_many.data_ptr())
    torch.cuda.synchronize()
    d_one = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    many = d_many.view(nq, -1)
    for b in range(nq):
        gpu.scan_dev(d_sel[b].data_ptr(), d_one.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(many[b], d_one), f"query {b} of {nq}"


def test_first_dim_matches_oracle_multi_tile(oracle):
    """Two 64-row chunks and two 128-column tiles of the byte-plane database
    against the oracle's first_dim."""
    import torch

    prm = paper_preset(128, 256)
    rng = np.random.default_rng(12)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"fd-multi")
    sel = rng.integers(0, prm.q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64)
    want = cpu.first_dim(sel)
    d_in = torch.from_numpy(sel.view(np.int64)).cuda()
    d_out = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    gpu.first_dim_dev(d_in.data_ptr(), d_out.data_ptr())
    assert np.array_equal(d_out.cpu().numpy().view(np.uint64), want)


@pytest.mark.parametrize("stage", [1, 2, 3, 4, 5, 6, 7])
def test_secure_preset_stage_parity(oracle, stage):
    """SECURE_PARAMS (n1 = 4096): every intermediate equals the oracle's."""
    prm = secure_preset(2, 4)
    rng = np.random.default_rng(40 + stage)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"secure-stage")
    q = client.query(int(rng.integers(prm.capacity)), b"secure-stage-q")
    got = gpu.debug_stage(q, stage)
    want = cpu.debug_stage(q, stage)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"stage {stage}: {bad.size} residues differ, first at {bad[:8]}"


def test_secure_preset_answers(oracle):
    prm = secure_preset(4, 8)
    rng = np.random.default_rng(4097)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client, gpu, cpu = _setup(oracle, prm, records, b"secure-answer")
    for idx in (0, int(rng.integers(prm.capacity))):
        _check_answer(client, gpu, cpu, records, idx, b"secure-a-%d" % idx)
