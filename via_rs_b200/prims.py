"""Primitive operations on device buffers (include/via_gpu.h via_ntt_*_dev,
via_external_product_dev, via_key_switch_dev): the reference's NTT, external
product and key switch (after a monomial rotation), run by the answer path's
kernels. Pointers are device addresses (e.g. torch.Tensor.data_ptr())."""
from __future__ import annotations

import ctypes

from . import _lib
from .server import check


def ring(n: int, primes) -> _lib.RingDesc:
    primes = list(primes)
    q = (ctypes.c_uint64 * 2)(primes[0], primes[1] if len(primes) > 1 else 0)
    return _lib.RingDesc(n, len(primes), q)


def ntt_forward_dev(r: _lib.RingDesc, data_ptr: int, count: int, stream: int = 0) -> None:
    check(_lib.lib().via_ntt_forward_dev(ctypes.byref(r), ctypes.c_void_p(data_ptr), count, ctypes.c_void_p(stream)))


def ntt_inverse_dev(r: _lib.RingDesc, data_ptr: int, count: int, stream: int = 0) -> None:
    check(_lib.lib().via_ntt_inverse_dev(ctypes.byref(r), ctypes.c_void_p(data_ptr), count, ctypes.c_void_p(stream)))


def external_product_dev(r: _lib.RingDesc, base: int, levels: int, rgsw_ptr: int, rlwe_ptr: int, count: int,
                         out_ptr: int, stream: int = 0) -> None:
    check(_lib.lib().via_external_product_dev(ctypes.byref(r), base, levels, ctypes.c_void_p(rgsw_ptr),
                                              ctypes.c_void_p(rlwe_ptr), count, ctypes.c_void_p(out_ptr),
                                              ctypes.c_void_p(stream)))


def key_switch_dev(r: _lib.RingDesc, base: int, levels: int, key_ptr: int, rlwe_ptr: int, shifts_ptr: int, count: int,
                   out_ptr: int, stream: int = 0) -> None:
    check(_lib.lib().via_key_switch_dev(ctypes.byref(r), base, levels, ctypes.c_void_p(key_ptr),
                                        ctypes.c_void_p(rlwe_ptr), ctypes.c_void_p(shifts_ptr), count,
                                        ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)))
