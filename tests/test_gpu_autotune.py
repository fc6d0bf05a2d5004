"""The FirstDim scan autotuner (via_server_autotune).

Every candidate tile computes the same exact sums (checked against single-query
scans, which other tests pin to the oracle's first_dim); tuned tiles survive a
cache file; answers after tuning (graphs re-captured under the new tiles) still
equal the oracle's and recover the record; a service that tunes at creation
serves the same answers.
"""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.server import PublicKeys, Server

pytestmark = pytest.mark.gpu


def _server(oracle, rows, cols, seed):
    prm = paper_preset(rows, cols)
    rng = np.random.default_rng(seed)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"tune-%d" % seed)
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), records)
    return prm, rng, records, client, gpu


@pytest.mark.parametrize("nq", [1, 3, 24, 40])
def test_every_candidate_tile_is_exact(oracle, nq):
    import torch

    prm, rng, _, _, gpu = _server(oracle, 128, 256, 21)
    cands = gpu.scan_tile_candidates(nq)
    assert cands[0] == {"n_max": 0, "stages": 0, "order": 0}
    assert len(cands) >= 3
    sel = rng.integers(0, prm.q2, size=(nq, prm.num_rows * 2 * prm.n1), dtype=np.uint64)
    sel[0, : 4 * prm.n1] = prm.q2 - 1  # largest exact sums in the first columns
    d_sel = torch.from_numpy(sel.view(np.int64)).cuda()
    d_one = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    want = []
    for b in range(nq):
        gpu.scan_dev(d_sel[b].data_ptr(), d_one.data_ptr())
        torch.cuda.synchronize()
        want.append(d_one.clone())
    d_out = torch.empty(nq * prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    for tile in cands:
        gpu.set_scan_tile(nq, tile)
        d_out.fill_(-1)
        gpu.scan_many_dev(d_sel.data_ptr(), nq, d_out.data_ptr())
        torch.cuda.synchronize()
        got = d_out.view(nq, -1)
        for b in range(nq):
            assert torch.equal(got[b], want[b]), f"tile {tile}, query {b} of {nq}"
    gpu.set_scan_tile(nq, None)


def test_invalid_tile_rejected(oracle):
    from via_rs_b200.server import ViaError

    _, _, _, _, gpu = _server(oracle, 64, 128, 24)
    with pytest.raises(ViaError):
        gpu.set_scan_tile(8, {"n_max": 40, "stages": 3, "order": 0})  # not 16, 32 or 48
    with pytest.raises(ViaError):
        gpu.set_scan_tile(1, {"n_max": 16, "stages": 3, "order": 0})  # one query has no column tiles
    with pytest.raises(ViaError):
        gpu.set_scan_tile(8, {"n_max": 48, "stages": 6, "order": 0})  # over the shared-memory limit


def test_autotune_cache_and_answers(oracle, tmp_path):
    prm, rng, records, client, gpu = _server(oracle, 64, 128, 22)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, records)
    idx = [int(x) for x in rng.integers(prm.capacity, size=3)]
    qs = [client.query(i, b"tune-q%d" % k) for k, i in enumerate(idx)]
    before = gpu.answer(qs[0])  # captures the one-query graph under the default tile

    cache = str(tmp_path / "scan_tiles.txt")
    first = gpu.autotune([1, 2, 3], cache)
    assert [e["batch"] for e in first] == [1, 2, 3]
    for e in first:
        assert e["candidates"] >= 2
        assert 0 < e["ms"] <= e["default_ms"]
    again = gpu.autotune([1, 2, 3], cache)
    for a, b in zip(first, again):
        assert b["candidates"] == 0, "the second call reads the cache file"
        assert b["tile"] == a["tile"]
    assert len(open(cache).read().splitlines()) == 3

    after = gpu.answer(qs[0])
    assert np.array_equal(after[0], before[0]) and np.array_equal(after[1], before[1])
    masks, bodies = gpu.answer_many(np.stack(qs))
    for k, i in enumerate(idx):
        cm, cb = cpu.answer(qs[k])
        assert np.array_equal(masks[k], cm) and np.array_equal(bodies[k], cb), f"query {k}"
        assert np.array_equal(client.recover(masks[k], bodies[k]), records[i])


def test_service_tunes_at_creation(oracle):
    from via_rs_b200.service import Service

    prm, rng, records, client, gpu = _server(oracle, 64, 128, 23)
    idx = [int(x) for x in rng.integers(prm.capacity, size=6)]
    qs = [client.query(i, b"svc-tune-%d" % k) for k, i in enumerate(idx)]
    alone = [gpu.answer(q) for q in qs]
    svc = Service(gpu, lanes=2, max_batch=4, warm=True, autotune=True)
    try:
        tuning = svc.tuning()
        assert [e["batch"] for e in tuning] == [1, 2, 4]
        assert all(e["candidates"] >= 2 for e in tuning)
        tickets = [svc.submit(q) for q in qs]
        for k, t in enumerate(tickets):
            m, b = svc.wait(t)
            assert np.array_equal(m, alone[k][0]) and np.array_equal(b, alone[k][1]), f"request {k}"
            assert np.array_equal(client.recover(m, b), records[idx[k]])
    finally:
        svc.close()
