"""The gadget decomposition the kernels run (exact integer scaling by invariant
divisors, balanced digits) against the oracle's gadget_scale_into /
gadget_extract_lsb_into, on the host: every gadget of every preset, with the
boundary coefficients (0, 1, Q/2, Q/2 + 1, Q - 1) and seeded random ones."""
import ctypes

import numpy as np
import pytest

from via_rs_b200 import _lib
from via_rs_b200.params import PAPER_Q1, PAPER_Q2, PAPER_Q3, SECURE_Q1

CASES = [
    (PAPER_Q1, 18, 18),      # cascade and conversion key (paper)
    (PAPER_Q1, 55879, 2),    # DMux
    ((PAPER_Q2,), 81, 2),    # CMux / CRot
    ((PAPER_Q2,), 18, 18),   # VIA-B repack at q2
    ((PAPER_Q3,), 8, 8),     # ring-switch key
    (SECURE_Q1, 18, 18),
    (SECURE_Q1, 18073, 2),
    ((PAPER_Q2,), 307, 2),
    ((PAPER_Q3,), 4, 8),
    ((1 << 40,), 2, 40),     # toy
    ((1 << 40,), 4, 20),
    ((1 << 32,), 4, 20),
    ((1 << 36,), 64, 7),     # n8
    ((1 << 16,), 4, 8),
]


def _coeffs(q, n, seed):
    Q = 1
    for x in q:
        Q *= x
    ints = [0, 1, 2, Q // 2 - 1, Q // 2, Q // 2 + 1, Q - 2, Q - 1]
    rng = np.random.default_rng(seed)
    ints += [int(v) for v in rng.integers(0, 2**62, size=n)] if Q > 2**62 else [int(v) for v in rng.integers(0, Q, size=n)]
    ints += [(int(a) << 62 | int(b)) % Q for a, b in zip(rng.integers(0, 2**62, size=n), rng.integers(0, 2**62, size=n))]
    out = np.array([[v % qi for qi in q] for v in ints], dtype=np.uint64)
    return out


@pytest.mark.parametrize("q,base,L", CASES)
def test_device_gadget_matches_oracle(oracle, q, base, L):
    coeffs = _coeffs(q, 20000, base + L)
    want = oracle.gadget_digits(q, base, L, coeffs)
    got = np.zeros(want.size, dtype=np.int64)
    rc = _lib.lib().via_gadget_digits_host(q[0], q[1] if len(q) > 1 else 0, base, L,
                                           coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), coeffs.shape[0],
                                           got.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    assert rc == 0, _lib.lib().via_last_error()
    got = got.reshape(want.shape)
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert bad.size == 0, f"{bad.size} coefficients differ, first {coeffs[bad[:3]]}: {got[bad[:3]]} vs {want[bad[:3]]}"
