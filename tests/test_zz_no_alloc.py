"""The no-allocation FirstDim scan against the regular one, through the C ABI.

via_first_dim_scan_static serves callers that cannot call cudaMalloc (for
example code running while a CUDA graph is being captured, or a host whose
device allocator belongs to another runtime): its scratch is a static device
array, so the call allocates nothing. It must give exactly the result of
via_first_dim_scan_dev, whose scratch is the server's own workspace, and keep
giving it on later calls, since every call reuses the same static array.
"""
import ctypes

import numpy as np
import pytest

from via_rs_b200 import _lib
from via_rs_b200.params import paper_preset
from via_rs_b200.server import DeviceError, PublicKeys, Server, check

pytestmark = pytest.mark.gpu


def _server(prm, seed):
    rng = np.random.default_rng(seed)
    q = min(prm.q1)
    keys = PublicKeys(rng.integers(0, q, size=prm.cascade_key_len, dtype=np.uint64),
                      rng.integers(0, q, size=prm.conv_key_len, dtype=np.uint64),
                      rng.integers(0, prm.q3, size=prm.rsk_len, dtype=np.uint64))
    records = rng.integers(0, 16, size=(prm.capacity, prm.n_rec), dtype=np.uint64)
    return Server.setup(prm, keys, records)


def test_static_scan_matches_workspace_scan_twice():
    import torch

    L = _lib.lib()
    prm = paper_preset(256, 64)  # I * 2 * n1 = 2^20: the largest shape the static scratch holds
    server = _server(prm, 5)
    rng = np.random.default_rng(6)
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    for call in range(2):  # a second call must not see the first call's scratch
        sel = torch.from_numpy(rng.integers(0, prm.q2, size=prm.num_rows * 2 * prm.n1, dtype=np.uint64)
                               .view(np.int64)).cuda()
        want = torch.empty(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
        got = torch.full_like(want, -1)
        check(L.via_first_dim_scan_dev(server._h, ctypes.c_void_p(sel.data_ptr()), ctypes.c_void_p(want.data_ptr()),
                                       sp))
        check(L.via_first_dim_scan_static(server._h, ctypes.c_void_p(sel.data_ptr()),
                                          ctypes.c_void_p(got.data_ptr()), sp))
        torch.cuda.synchronize()
        # Integer path: results must be identical (tolerance 0).
        assert torch.equal(got, want), f"call {call}: static-scratch scan differs"
    server.close()


def test_static_scan_rejects_shapes_beyond_its_scratch():
    import torch

    L = _lib.lib()
    prm = paper_preset(512, 8)  # I * 2 * n1 = 2^21 > 2^20
    server = _server(prm, 7)
    sel = torch.zeros(prm.num_rows * 2 * prm.n1, dtype=torch.int64, device="cuda")
    out = torch.zeros(prm.num_cols * 2 * prm.n1, dtype=torch.int64, device="cuda")
    with pytest.raises(DeviceError, match="static scratch"):
        check(L.via_first_dim_scan_static(server._h, ctypes.c_void_p(sel.data_ptr()),
                                          ctypes.c_void_p(out.data_ptr()), None))
    server.close()
