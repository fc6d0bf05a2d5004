"""Failure paths of the device answer path, made to happen without faulting the GPU.

The reference's error contract (crates/via-protocol/src/error.rs:20-64) is a
status per call. The device path adds VIA_ERR_TIMEOUT (a bounded wait ran out)
and VIA_ERR_BUSY (the serving queue is full). Every case here is produced on
purpose by the host or by the scan's test hook, and the context stays usable:
  * the FirstDim scan's bounded waits: via_server_set_scan_fault makes the
    epilogue wait on a barrier that nothing completes, for a few milliseconds;
    the CTAs abort after their copies and MMAs in flight have landed, and the
    synchronous calls and service requests report VIA_ERR_TIMEOUT. Turning the
    hook off clears the error word, and the next answers equal the oracle's;
  * via_service_wait with a limit shorter than the request takes;
  * via_service_submit into a full queue.
"""
import numpy as np
import pytest

from via_rs_b200.params import paper_preset
from via_rs_b200.server import DeviceError, PublicKeys, Server
from via_rs_b200.service import Service

pytestmark = pytest.mark.gpu

VIA_ERR_TIMEOUT = 103
VIA_ERR_BUSY = 104


def _setup(oracle, rows=4, cols=8, seed=51):
    prm = paper_preset(rows, cols)
    rng = np.random.default_rng(seed)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    client = oracle.Client(prm, b"failures-%d" % seed)
    keys = PublicKeys(client.cascade_key, client.conv_key, client.rsk)
    gpu = Server.setup(prm, keys, records)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, records)
    return prm, rng, records, client, gpu, cpu


def test_scan_wait_runs_out_and_handle_recovers(oracle):
    import torch

    prm, rng, records, client, gpu, cpu = _setup(oracle)
    sel = torch.from_numpy(rng.integers(0, prm.q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64)
                           .view(np.int64)).cuda()
    out = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    idx = int(rng.integers(prm.capacity))
    q = client.query(idx, b"fail-q")

    gpu.set_scan_fault(2000)  # 2 ms, then the wait gives up
    with pytest.raises(DeviceError) as e:
        gpu.first_dim_dev(sel.data_ptr(), out.data_ptr())
    assert e.value.code == VIA_ERR_TIMEOUT and "bounded device wait" in str(e.value)
    with pytest.raises(DeviceError) as e:
        gpu.answer(q)  # the answer graph is re-captured with the hook and runs out the same way
    assert e.value.code == VIA_ERR_TIMEOUT

    gpu.set_scan_fault(0)  # off again; the error word is cleared
    gm, gb = gpu.answer(q)
    cm, cb = cpu.answer(q)
    assert np.array_equal(gm, cm) and np.array_equal(gb, cb), "answer after recovery differs from the oracle"
    assert np.array_equal(client.recover(gm, gb), records[idx])
    gpu.close()


def test_service_reports_scan_timeouts_per_request(oracle):
    prm, rng, records, client, gpu, cpu = _setup(oracle, seed=52)
    qs = [client.query(int(i), b"svc-fail-%d" % k) for k, i in enumerate(rng.integers(prm.capacity, size=3))]
    gpu.set_scan_fault(2000)
    svc = Service(gpu, lanes=1, max_batch=4)
    try:
        tickets = [svc.submit(q) for q in qs]
        for t in tickets:
            with pytest.raises(DeviceError) as e:
                svc.wait(t, timeout_ms=60000)
            assert e.value.code == VIA_ERR_TIMEOUT
        assert svc.stats()["failed"] == len(qs)
    finally:
        svc.close()
    gpu.set_scan_fault(0)
    svc = Service(gpu, lanes=1, max_batch=4)
    try:
        m, b = svc.wait(svc.submit(qs[0]), timeout_ms=60000)
    finally:
        svc.close()
    cm, cb = cpu.answer(qs[0])
    assert np.array_equal(m, cm) and np.array_equal(b, cb)
    gpu.close()


def test_service_wait_limit_and_full_queue(oracle):
    prm, rng, records, client, gpu, cpu = _setup(oracle, rows=64, cols=256, seed=53)
    q = client.query(3, b"svc-wait")
    svc = Service(gpu, lanes=1, max_batch=1, max_pending=1)
    try:
        t = svc.submit(q)
        with pytest.raises(DeviceError) as e:
            svc.wait(t, timeout_ms=0)  # an answer takes milliseconds; a zero limit runs out first
        assert e.value.code == VIA_ERR_TIMEOUT
        m, b = svc.wait(t, timeout_ms=60000)  # the ticket stays valid
        assert np.array_equal(client.recover(m, b), records[3])
        # One request on the lane and one queued: further submits are refused
        # until the queue drains.
        accepted, busy = [], 0
        for _ in range(64):
            try:
                accepted.append(svc.submit(q))
            except DeviceError as err:
                assert err.code == VIA_ERR_BUSY
                busy += 1
        assert busy > 0, "a queue of one request never reported VIA_ERR_BUSY"
        for t in accepted:
            m, b = svc.wait(t, timeout_ms=60000)
            assert np.array_equal(client.recover(m, b), records[3])
    finally:
        svc.close()
    gpu.close()
