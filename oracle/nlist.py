"""ORACLE (test infrastructure only): brute-force typed neighbour list.

Restates the reference's neighbour-list semantics:
  * canonicalisation  ``(coord % box) * (ref/box) * (1 - 5e-7)`` in float32,
    then a stable sort by type (deepmd_jax/md_utils.py:364-373,
    deepmd_jax/utils.py:329-352);
  * the pair test of jax_md.partition.neighbor_list (third-party, unpinned git
    HEAD per setup.py:13, not vendored): displacement
    ``mod(Ri - Rj + L/2, L) - L/2`` (jax_md.space.periodic), squared distance
    summed in float32, kept if ``d2 < cutoff^2`` and ``j != i``;
  * the typed split ``get_nm`` (md_utils.py:431-459): per neighbour type the
    k smallest indices in ascending order, converted to type-local indices,
    padding value N (total atoms), last column dropped, overflow flagged when
    the last column is a real neighbour;
  * the capacity rule of ``allocate_fn`` (md_utils.py:394-403).

Parity status: unpinned at the one-ulp level — the summation order of the
three squared components inside jax_md is not visible here; this restatement
uses ((dx^2 + dy^2) + dz^2).  ``boundary_pairs`` reports how many pairs sit
within one ulp of the cutoff so a test can show the sets do not depend on it.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def jnp_mod(x, y):
    """jnp.mod / jnp.remainder semantics: fmod, then add y where the signs differ."""
    x = np.asarray(x)
    y = np.asarray(y, dtype=x.dtype)
    r = np.fmod(x, y)
    fix = (r != 0) & ((r < 0) != (y < 0))
    return np.where(fix, r + y, r).astype(x.dtype)


def canonicalize(coord, box, type_idx, ref_box=None):
    """float32 canonical coordinates in type-sorted order."""
    box32 = np.asarray(box, f32)
    ref = box32 if ref_box is None else np.asarray(ref_box, f32)
    scale = (ref / box32).astype(f32)
    c = jnp_mod(np.asarray(coord, f32), box32) * scale
    c = (c * f32(1 - 5e-7)).astype(f32)
    perm = np.argsort(np.asarray(type_idx), kind="stable")
    return c[perm]


def cutoff_sq(rcut_plus_skin, ref_box=None, box=None):
    """float32 square of the cutoff as jax_md receives it:
    rcut * max(ref/box) is a float32 scalar, squared in float32."""
    scale = f32(1.0) if ref_box is None else np.max(np.asarray(ref_box, f32) / np.asarray(box, f32)).astype(f32)
    c = f32(rcut_plus_skin) * scale
    return f32(c * c)


def pair_d2(ci, cj, L):
    """float32 min-image squared distance, centre minus neighbour."""
    L = np.asarray(L, f32)
    half = (L * f32(0.5)).astype(f32)
    d = jnp_mod((ci - cj).astype(f32) + half, L) - half
    d = d.astype(f32)
    return ((d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]).astype(f32)


def neighbor_sets(c, L, rc2, chunk=512):
    """All j != i with d2 < rc2 for canonical coords c (N,3) float32.
    Returns list of sorted int arrays (global sorted index)."""
    N = c.shape[0]
    out = []
    for s in range(0, N, chunk):
        ci = c[s:s + chunk]
        d2 = pair_d2(ci[:, None, :], c[None, :, :], L)
        m = d2 < rc2
        for k in range(ci.shape[0]):
            m[k, s + k] = False
            out.append(np.nonzero(m[k])[0].astype(np.int64))
    return out


def boundary_pairs(c, L, rc2, chunk=512):
    """Number of (i, j) pairs whose float32 d2 lies within one ulp of rc2."""
    lo = np.nextafter(rc2, f32(0))
    hi = np.nextafter(rc2, f32(np.inf))
    n = 0
    for s in range(0, c.shape[0], chunk):
        d2 = pair_d2(c[s:s + chunk, None, :], c[None, :, :], L)
        n += int(((d2 >= lo) & (d2 <= hi)).sum())
    return n


def typed_nlist(c, L, rc2, type_count, sel):
    """Typed block neighbour list (N, sum(sel)) int32 in the reference's
    nbrs_nm semantics (type-local ascending indices, pad N) plus the per-type
    neighbour counts (N, ntypes) and the overflow flag (any count > sel_j)."""
    N = c.shape[0]
    sets = neighbor_sets(c, L, rc2)
    offs = np.concatenate([[0], np.cumsum(type_count)])
    col = np.concatenate([[0], np.cumsum(sel)])
    out = np.full((N, col[-1]), N, dtype=np.int32)
    counts = np.zeros((N, len(sel)), dtype=np.int64)
    for i, s in enumerate(sets):
        for j in range(len(sel)):
            nb = s[(s >= offs[j]) & (s < offs[j + 1])] - offs[j]
            counts[i, j] = len(nb)
            k = min(len(nb), sel[j])
            out[i, col[j]:col[j] + k] = nb[:k]
    overflow = bool((counts > np.asarray(sel)[None, :]).any())
    return out, counts, overflow


def knbr_rule(max_counts, buffer_ratio=1.2):
    """Capacity rule of allocate_fn (md_utils.py:394-403); returns knbr
    (the slice kept is knbr - 1 columns)."""
    k = np.asarray(max_counts, float)
    knbr = np.where(k == 0, 1, 1 + (k * buffer_ratio + np.maximum(20 - k, 0) * max(buffer_ratio - 1.2, 0)))
    return knbr.astype(int)


def max_drift(c_now, c_ref, L):
    """max over atoms of the min-image displacement norm (utils.py:11-18,
    md.py:697-704), float32."""
    L = np.asarray(L, f32)
    d = jnp_mod((c_now - c_ref).astype(f32) - L / 2, L) - L / 2
    return float(np.sqrt((d.astype(f32) ** 2).sum(-1)).max())
