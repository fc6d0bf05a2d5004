"""Host logic of the mixed VIA-C / VIA-B service (via_rs_b200/mixed.py). No GPU needed.

A VIA-B request of m indices goes to the smallest power-of-two batch size T >= m that the
record-fit rule admits at n2 = 512 (crates/via-protocol/src/presets.rs:170-176); the client
pads it to T (crates/via-client/src/client.rs:256-300). The bench's mixed stream is a seeded
Poisson process with log-uniform VIA-B sizes.
"""
import numpy as np
import pytest

from via_rs_b200.mixed import POW2_BATCH_SIZES, _lane_queries, poisson_mix, via_b_route


def test_route_is_smallest_power_of_two_batch():
    assert POW2_BATCH_SIZES == (2, 4, 8, 16, 32, 64, 128, 256)
    for m in range(1, 257):
        t = via_b_route(m)
        assert t in POW2_BATCH_SIZES and t >= m
        assert t == 2 or t // 2 < m  # no smaller batch holds m
    with pytest.raises(ValueError):
        via_b_route(257)
    assert via_b_route(5, batch_sizes=(8, 256)) == 8
    assert via_b_route(9, batch_sizes=(256, 8)) == 256


def test_lane_sizes():
    assert _lane_queries("c", 64) == 64
    assert _lane_queries(2, 64) == 16  # small VIA-B routes keep lanes of at least 16 queries
    assert _lane_queries(32, 64) == 32
    assert _lane_queries(256, 64) == 64  # capped at max_batch


def test_poisson_mix_is_seeded_and_well_formed():
    a = poisson_mix(2000, 4.0, seed=22)
    assert a == poisson_mix(2000, 4.0, seed=22)
    assert a != poisson_mix(2000, 4.0, seed=23)
    gaps = np.array([g for g, _, _ in a])
    assert (gaps >= 0).all() and abs(gaps.mean() - 0.25) < 0.03  # rate 4/s
    kinds = [k for _, k, _ in a]
    assert abs(kinds.count("c") / len(kinds) - 0.5) < 0.05
    sizes = np.array([m for _, k, m in a if k == "b"])
    assert sizes.min() >= 1 and sizes.max() <= 256
    # log-uniform: about as many requests below 16 as from 16 to 256
    assert 0.35 < (sizes < 16).mean() < 0.65
    assert all(m == 1 for _, k, m in a if k == "c")
    only_c = poisson_mix(100, 1.0, seed=1, via_c_fraction=1.0)
    assert all(k == "c" for _, k, _ in only_c)
    small = poisson_mix(500, 1.0, seed=2, via_c_fraction=0.0, max_indices=8)
    assert max(m for _, _, m in small) <= 8
