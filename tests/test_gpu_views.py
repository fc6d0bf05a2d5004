"""One prepared database read at several record degrees (via_server_view), VIA-B
batches larger than a workspace (chunked prefix), and a mixed Poisson stream of
VIA-C queries and VIA-B batches of 1..256 indices served from one copy of the
database, every answer equal to the answer given alone and every record
recovered."""
import time

import numpy as np
import pytest

from via_rs_b200.mixed import POW2_BATCH_SIZES, MixedService, poisson_mix, via_b_route
from via_rs_b200.params import paper_preset
from via_rs_b200.server import PublicKeys, Server

pytestmark = pytest.mark.gpu


def _cells(prm, records):
    """VIA-C records [I*J*d][n_rec] -> cells [I*J][n1] (setup_db.rs:39-75)."""
    IJ, d = prm.num_rows * prm.num_cols, prm.n1 // prm.n_rec
    cells = np.zeros((IJ, prm.n1), dtype=np.uint64)
    for k in range(d):
        cells[:, k::d] = records[k * IJ:(k + 1) * IJ]
    return cells


def _view_records(prm_view, cells):
    """The records of degree prm_view.n_rec that the same cells hold."""
    IJ, d = cells.shape[0], prm_view.n1 // prm_view.n_rec
    return np.concatenate([cells[:, k::d] for k in range(d)], axis=0)


def _base(oracle, rows, cols, seed):
    prm = paper_preset(rows, cols)
    rng = np.random.default_rng(seed)
    recs = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"views-%d" % seed)
    keys = PublicKeys(client.cascade_key, client.conv_key, client.rsk)
    return prm, recs, keys, Server.setup(prm, keys, recs)


def _client(oracle, prm, keys_seed):
    return oracle.Client(prm, keys_seed)


@pytest.mark.parametrize("n3", [64, 2])
def test_view_equals_dedicated_server(oracle, n3):
    prm, recs, keys, base = _base(oracle, 4, 8, 31)
    pv = prm.with_dims(prm.num_rows, prm.num_cols, n3)
    vrecs = _view_records(pv, _cells(prm, recs))
    client = oracle.Client(pv, b"views-31")
    vkeys = PublicKeys(client.cascade_key, client.conv_key, client.rsk)
    view = base.view(n3, vkeys)
    dedicated = Server.setup(pv, vkeys, vrecs)
    T = pv.n2 // pv.n_rec
    rng = np.random.default_rng(n3)
    idx = [int(i) for i in rng.integers(pv.capacity, size=T)]
    qs = client.batch_query(idx, b"view-q")
    vm, vb = view.answer_batch(qs)
    dm, db = dedicated.answer_batch(qs)
    assert np.array_equal(vm, dm) and np.array_equal(vb, db), "view answer != dedicated server answer"
    got = client.recover_batch(vm, vb)
    for t, i in enumerate(idx):
        assert np.array_equal(got[t], vrecs[i]), (t, i)
    # The base keeps answering VIA-C queries from the shared cells.
    cc = oracle.Client(prm, b"views-31")
    i0 = int(rng.integers(prm.capacity))
    m, b = base.answer(cc.query(i0, b"base-q"))
    assert np.array_equal(cc.recover(m, b), recs[i0])


def test_view_outlives_base(oracle):
    prm, recs, keys, base = _base(oracle, 2, 4, 32)
    view = base.view(prm.n2)  # a VIA-C view with the base's keys
    base.close()
    client = oracle.Client(prm, b"views-32")
    q = client.query(5, b"outlive")
    m, b = view.answer(q)
    assert np.array_equal(client.recover(m, b), recs[5])


def test_t256_batch_in_chunks_through_service(oracle):
    """A lane whose workspace holds fewer than T = 256 queries answers the batch
    in chunks; the answer equals the direct answer_batch."""
    from via_rs_b200.service import Service, workspace_bytes

    prm, recs, keys, base = _base(oracle, 2, 4, 33)
    pv = prm.with_dims(2, 4, 2)
    client = oracle.Client(pv, b"views-33")
    view = base.view(2, PublicKeys(client.cascade_key, client.conv_key, client.rsk))
    vrecs = _view_records(pv, _cells(prm, recs))
    qbytes = pv.n_lwe * pv.lwe_len * 8
    budget = workspace_bytes(view, 48) + 256 * qbytes + (1 << 20)  # one lane of ~48 queries
    svc = Service(view, lanes=1, hbm_budget=budget)
    try:
        assert svc.stats()["batch_cap"] == 1
        rng = np.random.default_rng(5)
        idx = [int(i) for i in rng.integers(pv.capacity, size=256)]
        qs = client.batch_query(idx, b"chunks")
        m, b = svc.wait(svc.submit(qs))
    finally:
        svc.close()
    dm, db = view.answer_batch(qs)
    assert np.array_equal(m, dm) and np.array_equal(b, db)
    got = client.recover_batch(m, b)
    for t, i in enumerate(idx):
        assert np.array_equal(got[t], vrecs[i]), (t, i)


def test_mixed_poisson_stream(oracle):
    """Seeded Poisson arrivals of VIA-C queries and VIA-B requests of 1..256
    indices (log-uniform), each padded to the smallest power-of-two batch size
    T >= m; every answer equals the answer given alone and recovers the
    requested records."""
    prm, recs, keys, base = _base(oracle, 4, 8, 34)
    cells = _cells(prm, recs)
    clients = {"c": oracle.Client(prm, b"views-34")}
    records = {"c": recs}
    for t in POW2_BATCH_SIZES:
        pv = prm.with_dims(prm.num_rows, prm.num_cols, prm.n2 // t)
        clients[t] = oracle.Client(pv, b"views-34")
        records[t] = _view_records(pv, cells)
    mix = MixedService(base, lanes=2, max_batch=8, warm=True, autotune=False)
    try:
        rng = np.random.default_rng(35)
        plan = []
        for k, (gap, kind, m) in enumerate(poisson_mix(14, 40.0, seed=36)):
            if kind == "c":
                i = int(rng.integers(prm.capacity))
                plan.append((gap, "c", [i], 1, clients["c"].query(i, b"mix-%d" % k)))
            else:
                t = via_b_route(m)
                idx = [int(x) for x in rng.integers(records[t].shape[0], size=t)]  # m real + t - m padding
                plan.append((gap, t, idx, m, clients[t].batch_query(idx, b"mix-%d" % k)))
        handles = []
        for gap, route, idx, m, q in plan:
            time.sleep(gap)
            handles.append(mix.submit(route, q))
        results = [mix.wait(h) for h in handles]
        for (gap, route, idx, m, q), (am, ab) in zip(plan, results):
            srv = mix.servers[route]
            if route == "c":
                alone = srv.answer(q)
                assert np.array_equal(clients["c"].recover(am, ab), records["c"][idx[0]])
            else:
                alone = srv.answer_batch(q)
                got = clients[route].recover_batch(am, ab)
                for t in range(m):
                    assert np.array_equal(got[t], records[route][idx[t]]), (route, t)
            assert np.array_equal(am, alone[0]) and np.array_equal(ab, alone[1]), f"route {route}: mixed != alone"
        lat = mix.latencies()
        assert sum(len(v) for v in lat.values()) == len(plan)
    finally:
        mix.close()
