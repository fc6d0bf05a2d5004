"""The packed top byte plane of the scan's database chunks, checked on the host.

via_rs_b200/csrc/fd_tc.cuh: a 128 x 64 chunk holds each byte plane in the tensor-core
K-major core-matrix order, 16-byte group G = (kk * 16 + r / 8) * 8 + r % 8 holding rows
16 kk .. 16 kk + 15 of database column r. For q2 below 2^34 the top byte (at most 3) is
packed: quad Q of groups 4Q .. 4Q + 3 is four u32 words P_w, bits 8b + 2k of P_w holding
byte 4w + b of group 4Q + k. k_fd_planes ORs each group's bits into its quad; the scan's
unpack warp rebuilds group 4Q + k word w as (P_w >> 2k) & 0x03030303. This restates both
sides with numpy and checks that the rebuilt plane equals the plain one. No GPU needed.
"""
import numpy as np

FD_MT, FD_KC = 128, 64
PLANE = FD_MT * FD_KC


def plain_plane(top):
    """top[i][j] (64 x 128 bytes) -> the plane's 8192 bytes in core-matrix order."""
    out = np.zeros(PLANE, np.uint8)
    for kk in range(FD_KC // 16):
        for r in range(FD_MT):
            g = (kk * (FD_MT // 8) + r // 8) * 8 + r % 8
            out[g * 16:(g + 1) * 16] = top[16 * kk:16 * kk + 16, r]
    return out


def packed_plane(top):
    """k_fd_planes: per (kk, r) thread, OR its group's two-bit fields into the quad words."""
    words = np.zeros(PLANE // 16, np.uint32)  # 128 quads x 4 words
    for kk in range(FD_KC // 16):
        for r in range(FD_MT):
            g = (kk * (FD_MT // 8) + r // 8) * 8 + r % 8
            col = top[16 * kk:16 * kk + 16, r].astype(np.uint32)
            for w in range(4):
                word = col[4 * w] | col[4 * w + 1] << 8 | col[4 * w + 2] << 16 | col[4 * w + 3] << 24
                words[(g >> 2) * 4 + w] |= (word & 0x03030303) << (2 * (g & 3))
    return words


def unpack(words):
    """The unpack warp: lane l of iteration i expands quad Q = l + 32 i into four groups."""
    out = np.zeros(PLANE, np.uint8)
    for lane in range(32):
        for i in range(PLANE // 4 // 16 // 32):
            q = lane + 32 * i
            for k in range(4):
                for w in range(4):
                    word = (int(words[q * 4 + w]) >> (2 * k)) & 0x03030303
                    out[(4 * q + k) * 16 + 4 * w:(4 * q + k) * 16 + 4 * w + 4] = \
                        [(word >> (8 * b)) & 0xFF for b in range(4)]
    return out


def test_unpacked_plane_equals_plain_plane():
    rng = np.random.default_rng(2)
    q = 17175674881  # the paper preset's q2, below 2^34
    res = rng.integers(0, q, size=(FD_KC, FD_MT), dtype=np.uint64)
    res[0, :] = q - 1
    res[:, 0] = 0
    top = (res >> np.uint64(32)).astype(np.uint8)
    assert top.max() <= 3
    assert np.array_equal(unpack(packed_plane(top)), plain_plane(top))


def test_packed_chunk_sizes():
    # Four full planes and the packed one: 34816 bytes, a multiple of the 1024-byte
    # alignment the shared-memory stages keep; the expanded plane follows at that offset.
    chunk_p4 = 4 * PLANE + PLANE // 4
    assert chunk_p4 == 34816 and chunk_p4 % 1024 == 0
    assert (chunk_p4 + PLANE) % 1024 == 0
