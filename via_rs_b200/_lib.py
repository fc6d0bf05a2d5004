"""Loader for libvia_gpu.so, the CUDA implementation behind include/via_gpu.h.

There is no CPU fallback: if the library is missing or cannot load, every
entry point raises.
"""
import ctypes
import pathlib
import re

from .params import ViaParams

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libvia_gpu.so"
HEADER = HERE.parent / "include" / "via_gpu.h"

_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


class ViaPublicKeys(ctypes.Structure):
    _fields_ = [("cascade_key", _u64p), ("conv_key", _u64p), ("rsk", _u64p)]


class RingDesc(ctypes.Structure):
    """via_ring_desc: degree, limb count and primes of a ring."""
    _fields_ = [("n", ctypes.c_uint32), ("nl", ctypes.c_uint32), ("q", ctypes.c_uint64 * 2)]


class ScanTile(ctypes.Structure):
    """via_scan_tile: one FirstDim scan tile choice."""
    _fields_ = [("n_max", ctypes.c_uint32), ("stages", ctypes.c_uint32), ("order", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {"n_max": self.n_max, "stages": self.stages, "order": self.order}


class ScanTuning(ctypes.Structure):
    """via_scan_tuning: the autotuner's choice for one batch size."""
    _fields_ = [("batch", ctypes.c_uint32), ("tile", ScanTile), ("ms", ctypes.c_float), ("default_ms", ctypes.c_float),
                ("candidates", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {"batch": self.batch, "tile": self.tile.as_dict(), "ms": round(float(self.ms), 4),
                "default_ms": round(float(self.default_ms), 4), "candidates": self.candidates}


def declared_symbols() -> list:
    """Function names declared in include/via_gpu.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(via_[a-z0-9_]+)\s*\(", text)))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m via_rs_b200.build`")
    L = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.POINTER(ViaParams)
    L.via_last_error.restype = ctypes.c_char_p
    for name in ("via_lwe_len", "via_query_len", "via_cascade_key_len", "via_conv_key_len", "via_rsk_len"):
        f = getattr(L, name)
        f.restype = ctypes.c_uint64
        f.argtypes = [P]
    L.via_server_setup.restype = ctypes.c_int
    L.via_server_setup.argtypes = [P, ctypes.POINTER(ViaPublicKeys), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_void_p)]
    L.via_server_view.restype = ctypes.c_int
    L.via_server_view.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ViaPublicKeys),
                                  ctypes.POINTER(ctypes.c_void_p)]
    L.via_server_answer.restype = ctypes.c_int
    L.via_server_answer.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_uint64, _u64p, _u64p]
    L.via_server_destroy.restype = None
    L.via_server_destroy.argtypes = [ctypes.c_void_p]
    L.via_first_dim_dev.restype = ctypes.c_int
    L.via_first_dim_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.via_server_answer_dev.restype = ctypes.c_int
    L.via_server_answer_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
    L.via_first_dim_scan_dev.restype = ctypes.c_int
    L.via_first_dim_scan_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.via_server_answer_batch.restype = ctypes.c_int
    L.via_server_answer_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                          ctypes.c_void_p, ctypes.c_void_p]
    L.via_server_answer_batch_dev.restype = ctypes.c_int
    L.via_server_answer_batch_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.via_query_from_wire.restype = ctypes.c_int
    L.via_query_from_wire.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.c_uint64]
    L.via_server_answer_wire.restype = ctypes.c_int
    L.via_server_answer_wire.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                         ctypes.c_void_p]
    L.via_first_dim_scan_many_dev.restype = ctypes.c_int
    L.via_first_dim_scan_many_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                              ctypes.c_void_p]
    L.via_debug_stage.restype = ctypes.c_int
    L.via_debug_stage.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_uint64, ctypes.c_int, _u64p, ctypes.c_uint64]
    L.via_server_answer_many.restype = ctypes.c_int
    L.via_server_answer_many.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_uint64, ctypes.c_uint64, _u64p, _u64p]
    L.via_server_answer_many_dev.restype = ctypes.c_int
    L.via_server_answer_many_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.via_server_reserve.restype = ctypes.c_int
    L.via_server_reserve.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    L.via_server_transform_q2_dev.restype = ctypes.c_int
    L.via_server_transform_q2_dev.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                              ctypes.c_void_p]
    L.via_first_dim_scan_static.restype = ctypes.c_int
    L.via_first_dim_scan_static.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.via_server_autotune.restype = ctypes.c_int
    L.via_server_autotune.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64,
                                      ctypes.c_char_p, ctypes.POINTER(ScanTuning)]
    L.via_server_set_scan_tile.restype = ctypes.c_int
    L.via_server_set_scan_tile.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ScanTile)]
    L.via_server_set_scan_fault.restype = ctypes.c_int
    L.via_server_set_scan_fault.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
    L.via_scan_tile_candidates.restype = ctypes.c_uint64
    L.via_scan_tile_candidates.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ScanTile),
                                           ctypes.c_uint64]
    R = ctypes.POINTER(RingDesc)
    vp = ctypes.c_void_p
    for name in ("via_ntt_forward_dev", "via_ntt_inverse_dev"):
        f = getattr(L, name)
        f.restype = ctypes.c_int
        f.argtypes = [R, vp, ctypes.c_uint64, vp]
    L.via_external_product_dev.restype = ctypes.c_int
    L.via_external_product_dev.argtypes = [R, ctypes.c_uint64, ctypes.c_uint32, vp, vp, ctypes.c_uint64, vp, vp]
    L.via_key_switch_dev.restype = ctypes.c_int
    L.via_key_switch_dev.argtypes = [R, ctypes.c_uint64, ctypes.c_uint32, vp, vp, vp, ctypes.c_uint64, vp, vp]
    L.via_gadget_digits_host.restype = ctypes.c_int
    L.via_gadget_digits_host.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64,
                                         ctypes.POINTER(ctypes.c_int64)]
    L.via_kernel_launches.restype = ctypes.c_uint64
    L.via_kernel_launches.argtypes = []
    _lib = L
    return L
