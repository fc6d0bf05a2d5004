"""The no-allocation FirstDim scan, through the C ABI.

via_first_dim_scan_static serves callers that cannot call cudaMalloc: a host
whose device memory belongs to another runtime's allocator or a fixed pool, or a
latency-critical path that must not enter the allocator. Its scratch is a static
device array, so the call allocates nothing. It must give exactly the result of
via_first_dim_scan_dev (whose scratch is the server's own workspace) and of the
oracle's first_dim, and keep giving it on later calls, since every call reuses
the same static array.
"""
import ctypes

import numpy as np
import pytest

from via_rs_b200 import _lib
from via_rs_b200.params import paper_preset, toy_preset
from via_rs_b200.server import DeviceError, PublicKeys, Server, check

pytestmark = pytest.mark.gpu


def _setup(oracle, prm, seed):
    rng = np.random.default_rng(seed)
    client = oracle.Client(prm, b"no-alloc-%d" % seed)
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    keys = PublicKeys(client.cascade_key, client.conv_key, client.rsk)
    gpu = Server.setup(prm, keys, records)
    cpu = oracle.Server(prm, client.cascade_key, client.conv_key, client.rsk, records)
    return rng, gpu, cpu


@pytest.mark.parametrize("preset", ["paper", "toy"])
def test_static_scan_matches_workspace_scan_and_oracle_twice(oracle, preset):
    """Two calls in a row, each with fresh selection vectors: static scan ==
    workspace scan == oracle first_dim, residue for residue (integer path,
    tolerance 0). The paper case has I = 256 at n1 = 2048, the largest shape the
    static scratch holds; the toy case (schoolbook ring) needs no scratch."""
    import torch

    L = _lib.lib()
    prm = paper_preset(256, 32) if preset == "paper" else toy_preset(16, 16)
    rng, gpu, cpu = _setup(oracle, prm, 5)
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    for call in range(2):  # the second call must not see the first call's scratch
        sel = rng.integers(0, prm.q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64)
        want_cpu = cpu.first_dim(sel)
        d_sel = torch.from_numpy(sel.view(np.int64)).cuda()
        gpu.transform_q2_dev(d_sel.data_ptr(), prm.num_rows * 2, stream=stream.cuda_stream)
        want = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
        got = torch.full_like(want, -1)
        check(L.via_first_dim_scan_dev(gpu._h, ctypes.c_void_p(d_sel.data_ptr()),
                                       ctypes.c_void_p(want.data_ptr()), sp))
        check(L.via_first_dim_scan_static(gpu._h, ctypes.c_void_p(d_sel.data_ptr()),
                                          ctypes.c_void_p(got.data_ptr()), sp))
        stream.synchronize()
        assert torch.equal(got, want), f"call {call}: static-scratch scan differs from the workspace scan"
        gpu.transform_q2_dev(got.data_ptr(), prm.num_cols * 2, inverse=True, stream=stream.cuda_stream)
        stream.synchronize()
        got_coef = got.cpu().numpy().view(np.uint64)
        bad = np.nonzero(got_coef != want_cpu)[0]
        assert bad.size == 0, f"call {call}: {bad.size} residues differ from the oracle, first at {bad[:8]}"
    gpu.close()


def test_static_scan_rejects_shapes_beyond_its_scratch():
    import torch

    L = _lib.lib()
    prm = paper_preset(512, 8)  # 16 * I_pad * n1 = 2^24 bytes > the 8 MiB scratch
    rng = np.random.default_rng(7)
    q = min(prm.q1)
    keys = PublicKeys(rng.integers(0, q, size=prm.cascade_key_len, dtype=np.uint64),
                      rng.integers(0, q, size=prm.conv_key_len, dtype=np.uint64),
                      rng.integers(0, prm.q3, size=prm.rsk_len, dtype=np.uint64))
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    server = Server.setup(prm, keys, records)
    sel = torch.zeros(prm.num_rows * 2 * prm.n1, dtype=torch.int64, device="cuda")
    out = torch.zeros(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    with pytest.raises(DeviceError, match="static scratch"):
        check(L.via_first_dim_scan_static(server._h, ctypes.c_void_p(sel.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), None))
    server.close()
