"""The C-ABI library loads and exports every entry point include/via_gpu.h declares.

No compute calls: these run without a GPU.
"""
import ctypes

import pytest

from via_rs_b200 import _lib
from via_rs_b200.params import ViaParams, n8_preset, paper_preset, toy_preset


def test_library_exports_header_symbols():
    L = _lib.lib()
    syms = _lib.declared_symbols()
    assert "via_server_setup" in syms and "via_server_answer" in syms
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/via_gpu.h but not exported"


def test_params_struct_layout():
    # Offsets of the C struct (include/via_gpu.h) as ctypes lays it out.
    assert ctypes.sizeof(ViaParams) == 4 * 4 + 8 * 12 + 4 * 4
    assert ViaParams.num_rows.offset == 16
    assert ViaParams.l_query.offset == 16 + 8 * 12


@pytest.mark.parametrize("prm", [n8_preset(), toy_preset(), paper_preset()], ids=["n8", "toy", "paper"])
def test_buffer_lengths_agree(prm):
    L = _lib.lib()
    c = prm.to_c()
    assert L.via_lwe_len(ctypes.byref(c)) == prm.lwe_len
    assert L.via_query_len(ctypes.byref(c)) == prm.n_lwe
    assert L.via_cascade_key_len(ctypes.byref(c)) == prm.cascade_key_len
    assert L.via_conv_key_len(ctypes.byref(c)) == prm.conv_key_len
    assert L.via_rsk_len(ctypes.byref(c)) == prm.rsk_len


def test_paper_sizes():
    prm = paper_preset()
    assert prm.n_lwe == 44  # (8 + 12 + 2) bits x L_QUERY 2 at 1 GiB
    assert prm.cascade_key_len * 8 == 25_952_256  # the 24.75 MiB cascade key
    assert prm.capacity * prm.n_rec * 4 // 8 == 1 << 30  # 1 GiB of 4-bit records
