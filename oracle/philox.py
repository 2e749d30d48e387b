"""ORACLE (test infrastructure only): Philox4x32-10 counter-based generator
(Salmon, Moraes, Dror, Shaw, SC'11 "Parallel random numbers: as easy as
1, 2, 3") and the Box-Muller normals the device kernels draw from it.

Stream definition shared with deepmd-jax_b200/csrc/md_kernels.cu:
  key     = (seed & 0xffffffff, seed >> 32)
  counter = (q, step, tag, 0) for element block q (elements 4q .. 4q+3)
  u_a     = x_a * 2^-32 + 2^-33                      (a = 0..3, never 0)
  normals = sqrt(-2 ln u0) * (cos 2pi u1, sin 2pi u1),
            sqrt(-2 ln u2) * (cos 2pi u3, sin 2pi u3)
"""
from __future__ import annotations

import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)


def philox4x32(c0, c1, c2, c3, k0, k1, rounds=10):
    c0 = np.asarray(c0, np.uint32).copy()
    c1 = np.broadcast_to(np.asarray(c1, np.uint32), c0.shape).copy()
    c2 = np.broadcast_to(np.asarray(c2, np.uint32), c0.shape).copy()
    c3 = np.broadcast_to(np.asarray(c3, np.uint32), c0.shape).copy()
    k0 = np.uint32(k0)
    k1 = np.uint32(k1)
    with np.errstate(over="ignore"):
        for r in range(rounds):
            p0 = c0.astype(np.uint64) * M0
            p1 = c2.astype(np.uint64) * M1
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & MASK).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & MASK).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            k0 = np.uint32(k0 + W0)
            k1 = np.uint32(k1 + W1)
    return c0, c1, c2, c3


def normals(n, seed, step, tag):
    """n standard normals (float64) of the stream (seed, step, tag)."""
    nq = (n + 3) // 4
    q = np.arange(nq, dtype=np.uint32)
    k0 = seed & 0xFFFFFFFF
    k1 = (seed >> 32) & 0xFFFFFFFF
    x = philox4x32(q, step, tag, 0, k0, k1)
    u = [xa.astype(np.float64) * 2.0 ** -32 + 2.0 ** -33 for xa in x]
    r0 = np.sqrt(-2.0 * np.log(u[0]))
    r1 = np.sqrt(-2.0 * np.log(u[2]))
    out = np.stack([r0 * np.cos(2 * np.pi * u[1]), r0 * np.sin(2 * np.pi * u[1]),
                    r1 * np.cos(2 * np.pi * u[3]), r1 * np.sin(2 * np.pi * u[3])], axis=1)
    return out.reshape(-1)[:n]
