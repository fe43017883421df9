"""Philox4x32-10 counter-based generator (Salmon, Moraes, Dror & Shaw, SC'11).  TEST INFRASTRUCTURE.

Restated from the published algorithm so the oracle draws the same seeded perturbation as the
C++ host code (``afid-murphfi_b200/csrc/afid_host.cpp``, ``afid_philox_uniform``):

* counter = (n mod 2^32, n >> 32, 0, 0) for the global linear cell index n = k + nx*(j + nym*i);
* key     = (seed mod 2^32, seed >> 32);
* 10 rounds with multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl increments 0x9E3779B9 / 0xBB67AE85;
* uniform U = ((out0 << 21) | (out1 >> 11)) * 2^-53, a 53-bit double in [0, 1).
"""
from __future__ import annotations

import numpy as np

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = np.uint64(0x9E3779B9)
_W1 = np.uint64(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32(ctr: np.ndarray, key0: int, key1: int):
    """Vectorised Philox4x32-10.  ``ctr`` is (4, n) uint64 holding 32-bit words."""
    c0, c1, c2, c3 = (ctr[i].astype(np.uint64) for i in range(4))
    k0 = np.uint64(key0 & 0xFFFFFFFF)
    k1 = np.uint64(key1 & 0xFFFFFFFF)
    for r in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & _MASK, lo1, (hi0 ^ c3 ^ k1) & _MASK, lo0
        k0 = (k0 + _W0) & _MASK
        k1 = (k1 + _W1) & _MASK
    return c0, c1, c2, c3


def uniform_from_counter(n: np.ndarray, seed: int) -> np.ndarray:
    n = np.asarray(n, dtype=np.uint64)
    ctr = np.zeros((4,) + n.shape, dtype=np.uint64)
    ctr[0] = n & _MASK
    ctr[1] = n >> np.uint64(32)
    o0, o1, _, _ = philox4x32(ctr, seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    bits = (o0 << np.uint64(21)) | (o1 >> np.uint64(11))
    return bits.astype(np.float64) * (2.0 ** -53)


def uniform_cells(seed: int, nzm: int, nym: int, nx: int) -> np.ndarray:
    """U for every cell of a (nzm, nym, nx) array, keyed by n = k + nx*(j + nym*i)."""
    n = np.arange(nzm * nym * nx, dtype=np.uint64).reshape(nzm, nym, nx)
    return uniform_from_counter(n, seed)
