"""Primitive kernels on the GPU (via_ntt_*_dev, via_external_product_dev,
via_key_switch_dev) against the oracle, bit-exact.

The NTT's eval form is the reference's own (same root and order), so forward
outputs are compared directly. The last tests run the kernel micro-benchmark
sizes (65536 RNS polynomials of degree 2048; 16384 external products and key
switches) and check a seeded sample of each batch against the oracle (every
item is independent), plus the NTT round trip on the whole batch.
"""
import numpy as np
import pytest

from via_rs_b200 import prims
from via_rs_b200.params import PAPER_Q1, PAPER_Q2, PAPER_Q3, SECURE_Q1

pytestmark = pytest.mark.gpu

Q1 = tuple(PAPER_Q1)


def _dev_rand(torch, q, n, count, gen):
    """[count][nl][n] uniform residues on the device."""
    parts = [torch.randint(0, int(qi), (count, 1, n), dtype=torch.int64, device="cuda", generator=gen) for qi in q]
    return torch.cat(parts, dim=1).contiguous()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("q,n", [(Q1, 2048), ((PAPER_Q2,), 2048), ((PAPER_Q3,), 512), (tuple(SECURE_Q1), 4096),
                                 (Q1, 64), ((PAPER_Q2,), 2)])
def test_ntt_matches_oracle(oracle, q, n):
    import torch

    gen = torch.Generator(device="cuda").manual_seed(n + len(q))
    x = _dev_rand(torch, q, n, 24, gen)
    x0 = x.clone()
    r = prims.ring(n, q)
    prims.ntt_forward_dev(r, x.data_ptr(), 24)
    torch.cuda.synchronize()
    want = oracle.ntt(q, n, _host(x0))
    assert np.array_equal(_host(x), want), "forward NTT differs from the reference transform"
    prims.ntt_inverse_dev(r, x.data_ptr(), 24)
    torch.cuda.synchronize()
    assert torch.equal(x, x0)


@pytest.mark.parametrize("q,n,base,L", [(Q1, 2048, 55879, 2), ((PAPER_Q2,), 2048, 81, 2), (Q1, 256, 18, 3),
                                        (tuple(SECURE_Q1), 4096, 18073, 2)])
def test_external_product_matches_oracle(oracle, q, n, base, L):
    import torch

    gen = torch.Generator(device="cuda").manual_seed(7)
    count = 12
    rgsw = _dev_rand(torch, q, n, count * 2 * L * 2, gen)
    ct = _dev_rand(torch, q, n, count * 2, gen)
    ct[0].zero_()  # a zero mask: all-zero digits
    out = torch.empty_like(ct)
    prims.external_product_dev(prims.ring(n, q), base, L, rgsw.data_ptr(), ct.data_ptr(), count, out.data_ptr())
    want = oracle.external_product(q, n, base, L, _host(rgsw), _host(ct))
    assert np.array_equal(_host(out).reshape(-1), want)


@pytest.mark.parametrize("q,n,base,L", [(Q1, 2048, 18, 18), ((PAPER_Q2,), 1024, 18, 8), (Q1, 16, 18, 18)])
def test_key_switch_matches_oracle(oracle, q, n, base, L):
    import torch

    gen = torch.Generator(device="cuda").manual_seed(9)
    count = 10
    key = _dev_rand(torch, q, n, L * 2, gen)
    ct = _dev_rand(torch, q, n, count * 2, gen)
    shifts = np.array([0, 1, n - 1, n, n + 1, 2 * n - 1, 2 * n, 3 * n + 5, 7, 12345], dtype=np.uint64)
    d_shifts = torch.from_numpy(shifts.view(np.int64)).cuda()
    out = torch.empty_like(ct)
    prims.key_switch_dev(prims.ring(n, q), base, L, key.data_ptr(), ct.data_ptr(), d_shifts.data_ptr(), count,
                         out.data_ptr())
    want = oracle.key_switch(q, n, base, L, _host(key), _host(ct), shifts)
    assert np.array_equal(_host(out).reshape(-1), want)


def test_prims_reject_bad_rings():
    import torch

    from via_rs_b200.server import ViaError

    x = torch.zeros(2 * 64, dtype=torch.int64, device="cuda")
    with pytest.raises(ViaError):
        prims.ntt_forward_dev(prims.ring(64, (PAPER_Q2 + 2,)), x.data_ptr(), 1)  # not prime / not NTT-friendly
    with pytest.raises(ViaError):
        prims.ntt_forward_dev(prims.ring(48, (PAPER_Q2,)), x.data_ptr(), 1)  # not a power of two
    with pytest.raises(ViaError):
        prims.ntt_forward_dev(prims.ring(8192, (PAPER_Q2,)), x.data_ptr(), 1)  # above 4096


# ---- kernel micro-benchmark sizes (n = 2048 over the two q1 primes) --------

def _sample(count, k, seed):
    return np.sort(np.random.default_rng(seed).choice(count, size=k, replace=False))


def test_ntt_65536_polys(oracle):
    import torch

    count, n = 65536, 2048
    gen = torch.Generator(device="cuda").manual_seed(1)
    x = _dev_rand(torch, Q1, n, count, gen)
    x0 = x.clone()
    r = prims.ring(n, Q1)
    prims.ntt_forward_dev(r, x.data_ptr(), count)
    torch.cuda.synchronize()
    idx = _sample(count, 48, 2)
    want = oracle.ntt(Q1, n, _host(x0[idx]))
    assert np.array_equal(_host(x[idx]), want)
    prims.ntt_inverse_dev(r, x.data_ptr(), count)
    torch.cuda.synchronize()
    assert torch.equal(x, x0), "inverse(forward(x)) != x on the full batch"


def test_external_products_16384_pairs(oracle):
    import torch

    count, n, base, L = 16384, 2048, 55879, 2
    gen = torch.Generator(device="cuda").manual_seed(3)
    rgsw = _dev_rand(torch, Q1, n, count * 2 * L * 2, gen)
    ct = _dev_rand(torch, Q1, n, count * 2, gen)
    out = torch.empty_like(ct)
    prims.external_product_dev(prims.ring(n, Q1), base, L, rgsw.data_ptr(), ct.data_ptr(), count, out.data_ptr())
    idx = _sample(count, 32, 4)
    rg = rgsw.view(count, -1)[idx]
    cs = ct.view(count, -1)[idx]
    want = oracle.external_product(Q1, n, base, L, _host(rg), _host(cs))
    assert np.array_equal(_host(out.view(count, -1)[idx]).reshape(-1), want)


def test_key_switches_16384(oracle):
    import torch

    count, n, base, L = 16384, 2048, 18, 18
    gen = torch.Generator(device="cuda").manual_seed(5)
    key = _dev_rand(torch, Q1, n, L * 2, gen)
    ct = _dev_rand(torch, Q1, n, count * 2, gen)
    shifts = np.random.default_rng(6).integers(0, 2 * n, size=count, dtype=np.uint64)
    d_shifts = torch.from_numpy(shifts.view(np.int64)).cuda()
    out = torch.empty_like(ct)
    prims.key_switch_dev(prims.ring(n, Q1), base, L, key.data_ptr(), ct.data_ptr(), d_shifts.data_ptr(), count,
                         out.data_ptr())
    idx = _sample(count, 32, 7)
    want = oracle.key_switch(Q1, n, base, L, _host(key), _host(ct.view(count, -1)[idx]), shifts[idx])
    assert np.array_equal(_host(out.view(count, -1)[idx]).reshape(-1), want)
