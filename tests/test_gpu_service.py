"""The continuous-batching service: every answer is the same alone and in the mix.

A query answered alone through the service, the same query answered among many
others (batched with whatever was pending, several batches in flight on
separate lanes), and the direct single-answer call all return the same
residues, equal to the oracle's, and the client recovers the record.
"""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.server import PublicKeys, Server
from via_rs_b200.service import Service, workspace_bytes

pytestmark = pytest.mark.gpu


def _setup(oracle, rows, cols, n_rec, seed):
    prm = paper_preset(rows, cols, n_rec=n_rec)
    rng = np.random.default_rng(len(seed))
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, seed)
    gpu = Server.setup(prm, PublicKeys(client.cascade_key, client.conv_key, client.rsk), recs)
    return prm, recs, client, gpu


def test_results_same_alone_and_in_mix(oracle):
    prm, recs, client, gpu = _setup(oracle, 8, 16, 512, b"service-mix")
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, recs)
    rng = np.random.default_rng(3)
    idx = [int(i) for i in rng.integers(prm.capacity, size=24)]
    qs = [client.query(i, b"svc-%d" % k) for k, i in enumerate(idx)]
    svc = Service(gpu, lanes=2, max_batch=8)
    try:
        alone = svc.wait(svc.submit(qs[11]))
        tickets = [svc.submit(q) for q in qs]  # all at once: batched and overlapped
        mixed = [svc.wait(t) for t in tickets]
        st = svc.stats()
    finally:
        svc.close()
    assert np.array_equal(alone[0], mixed[11][0]) and np.array_equal(alone[1], mixed[11][1])
    for k, i in enumerate(idx):
        dm, db = gpu.answer(qs[k])
        assert np.array_equal(mixed[k][0], dm) and np.array_equal(mixed[k][1], db), k
        assert np.array_equal(client.recover(*mixed[k]), recs[i]), k
    cm, cb = cpu.answer(qs[11])
    assert np.array_equal(alone[0], cm) and np.array_equal(alone[1], cb)
    assert st["completed"] == 25 and st["failed"] == 0
    assert st["batches"] < 25 and st["mean_batch"] > 1.0, st
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_admission_by_hbm_budget(oracle):
    prm, recs, client, gpu = _setup(oracle, 4, 8, 512, b"service-budget")
    one = Service(gpu, lanes=1, max_batch=64)
    cap_free = one.stats()["batch_cap"]
    one.close()
    assert cap_free == 64
    # A budget for three queries per lane caps the batch; requests beyond it wait.
    probe = Service(gpu, lanes=2, max_batch=64, hbm_budget=2 * workspace_bytes(gpu, 3) + 1024)
    cap = probe.stats()["batch_cap"]
    idx = list(range(min(prm.capacity, 3 * cap + 1)))
    tickets = [probe.submit(client.query(i, b"b-%d" % i)) for i in idx]
    res = [probe.wait(t) for t in tickets]
    st = probe.stats()
    probe.close()
    assert cap == 3
    assert st["batches"] >= -(-len(idx) // cap)
    for k, i in enumerate(idx):
        assert np.array_equal(client.recover(*res[k]), recs[i])


def test_via_b_groups(oracle):
    prm, recs, client, gpu = _setup(oracle, 2, 2, 64, b"service-via-b")
    groups = [client.batch_query([int(x) for x in np.random.default_rng(g).integers(prm.capacity, size=8)],
                                 b"g%d" % g) for g in range(3)]
    svc = Service(gpu, lanes=2, max_batch=2)
    try:
        tickets = [svc.submit(q) for q in groups]
        res = [svc.wait(t) for t in tickets]
    finally:
        svc.close()
    for g, q in enumerate(groups):
        dm, db = gpu.answer_batch(q)
        assert np.array_equal(res[g][0], dm) and np.array_equal(res[g][1], db), g
