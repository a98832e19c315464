"""CPU restatement of the engine's device phonon generator (pn_rng 1) — TEST INFRASTRUCTURE ONLY.

The reference has no counterpart: it draws displacements on the host from mt19937_64 streams
(Spec::move_atoms, src/spec.hpp:85-127). The device generator replaces that serial sequence with
a counter-based one, so there is no reference output to pin; this module pins the generator to the
published Philox4x32-10 known-answer vectors instead (Salmon, Moraes, Dror and Shaw, "Parallel
random numbers: as easy as 1, 2, 3", SC'11, and the test vectors distributed with their Random123
library), and restates the Box-Muller step so that the device's displaced positions can be
checked value by value.
"""
from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_LO = np.uint64(0xFFFFFFFF)
_S32 = np.uint64(32)

# (counter, key, result) triples of Philox4x32-10 from the Random123 known-answer vectors
KAT = (
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff), (0xffffffff, 0xffffffff),
     (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
)


def philox4x32_10(ctr, key):
    """ctr [n, 4], key [n, 2] (uint32) -> [n, 4] uint32."""
    c = [np.asarray(ctr, dtype=np.uint32).reshape(-1, 4)[:, j].copy() for j in range(4)]
    k0, k1 = (np.asarray(key, dtype=np.uint32).reshape(-1, 2)[:, j].copy() for j in range(2))
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = M0 * c[0].astype(np.uint64)
            p1 = M1 * c[2].astype(np.uint64)
            hi0, lo0 = (p0 >> _S32).astype(np.uint32), (p0 & _LO).astype(np.uint32)
            hi1, lo1 = (p1 >> _S32).astype(np.uint32), (p1 & _LO).astype(np.uint32)
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
            k0 = k0 + W0
            k1 = k1 + W1
    return np.stack(c, axis=1)


def normals(n, seed, iconf):
    """The two standard normals (x, y) of atoms 0..n-1 in configuration iconf, float64."""
    i = np.arange(n, dtype=np.uint32)
    ctr = np.stack([i, np.full(n, iconf, np.uint32), np.zeros(n, np.uint32), np.zeros(n, np.uint32)], axis=1)
    key = np.stack([np.full(n, seed, np.uint32), np.zeros(n, np.uint32)], axis=1)
    r = philox4x32_10(ctr, key)
    u0 = (r[:, 0].astype(np.float64) + 0.5) * 2.0 ** -32
    u1 = (r[:, 1].astype(np.float64) + 0.5) * 2.0 ** -32
    rad = np.sqrt(-2.0 * np.log(u0))
    a = 6.283185307179586 * u1
    return rad * np.cos(a), rad * np.sin(a)


def displaced(xyz, sigma, seed, iconf, pn_x=True, pn_y=True):
    """Atoms (float32 x, y; z unchanged) of configuration iconf, as the device generator moves them."""
    xyz = np.asarray(xyz, dtype=np.float32).copy()
    nx, ny = normals(len(xyz), seed, iconf)
    s = np.asarray(sigma, dtype=np.float32)
    if pn_x:
        xyz[:, 0] = xyz[:, 0] + s * nx.astype(np.float32)
    if pn_y:
        xyz[:, 1] = xyz[:, 1] + s * ny.astype(np.float32)
    return xyz
