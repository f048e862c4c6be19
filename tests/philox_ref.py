"""Host restatement of the counter-based generator behind the library's GPU RNG
(cuRng32* / cuRng64*): Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel
random numbers: as easy as 1, 2, 3", SC 2011), with the library's stream layout and
float conversions.  Test infrastructure: it checks the device generator bit for bit
and rebuilds on the host the random draws of the device SPD generator (cu?latmc).

Layout: word i of a stream seeded with key (k0, k1) is word i mod 4 of
Philox4x32-10(counter = (b mod 2^32, b div 2^32, 0, 0), key), b = i div 4.  64-bit
values take two consecutive words, the first as the low half.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr, key):
    """ctr: uint32 array (m, 4); key: two ints.  Returns uint32 (m, 4)."""
    c = [np.asarray(ctr[:, i], dtype=np.uint64) for i in range(4)]
    k0, k1 = int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF
    for r in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = [hi1 ^ c[1] ^ np.uint64(k0), lo1, hi0 ^ c[3] ^ np.uint64(k1), lo0]
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return np.stack([x.astype(np.uint32) for x in c], axis=1)


def words(key, start_word: int, count: int) -> np.ndarray:
    """count consecutive 32-bit words of the stream from word start_word (a multiple
    of 4)."""
    assert start_word % 4 == 0
    b0 = start_word // 4
    nb = (count + 3) // 4
    b = np.arange(b0, b0 + nb, dtype=np.uint64)
    ctr = np.zeros((nb, 4), dtype=np.uint64)
    ctr[:, 0] = b & MASK
    ctr[:, 1] = b >> np.uint64(32)
    return philox4x32_10(ctr, key).reshape(-1)[:count]


def u64(key, start_block: int, count: int) -> np.ndarray:
    """count 64-bit values from Philox block start_block (two per block)."""
    w = words(key, 4 * start_block, 2 * count).astype(np.uint64)
    return w[0::2] | (w[1::2] << np.uint64(32))


def to_f32(x: np.ndarray, kind: str) -> np.ndarray:
    x = x.astype(np.uint64)
    if kind == "co":
        return ((x >> np.uint64(8)).astype(np.float64) * 2.0 ** -24).astype(np.float32)
    if kind == "oc":
        return (((x >> np.uint64(8)) + np.uint64(1)).astype(np.float64) * 2.0 ** -24).astype(np.float32)
    if kind == "oo":
        return (((x >> np.uint64(9)).astype(np.float64) + 0.5) * 2.0 ** -23).astype(np.float32)
    return ((x >> np.uint64(8)).astype(np.float32) / np.float32(16777215.0)).astype(np.float32)


def to_f64(y: np.ndarray, kind: str) -> np.ndarray:
    if kind == "co":
        return (y >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    if kind == "oc":
        return ((y >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53
    if kind == "oo":
        return ((y >> np.uint64(12)).astype(np.float64) + 0.5) * 2.0 ** -52
    return (y >> np.uint64(11)).astype(np.float64) / 9007199254740991.0
