"""Typed neighbour lists with the reference's interface
(deepmd_jax/md_utils.py:353-461), built on the device by dpb_nlist_build.

``typed_neighbor_list(box, type_idx, type_count, rcut, buffer_ratio)`` returns
an object with ``allocate(coord, box, knbr_override)`` and
``update(coord, typed_nbrs, box)``.  The list is held in one packed int32
array ``nbrs`` of shape (N, sum(knbr) - ntypes) in type-sorted atom order:
columns [col_j, col_j + knbr_j - 1) hold the type-j neighbours of each centre
as type-local indices, ascending, padded with N.  ``nbrs_nm[i][j]`` are the
views of that array the reference's model consumes: rows of centre type i,
columns of neighbour type j, shape (N_i, knbr_j - 1).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from types import SimpleNamespace

import numpy as np
import torch

from .engine import NeighborBuilder, _require_cuda, sort_by_type

MEASURE_CAPACITY = 256


def knbr_from_counts(max_counts, buffer_ratio):
    """Per-type capacity from the measured maximum neighbour counts
    (deepmd_jax/md_utils.py:394-403): 1 for an absent type, otherwise
    1 + count * buffer_ratio + max(20 - count, 0) * max(buffer_ratio - 1.2, 0)."""
    k = np.asarray(max_counts, dtype=np.int64)
    grown = 1 + (k * buffer_ratio + np.maximum(20 - k, 0) * max(buffer_ratio - 1.2, 0))
    return [int(x) for x in np.where(k == 0, 1, grown).astype(int)]


def to_nbrs_nm(nbrs, type_count, sel):
    """Views nbrs_nm[i][j] of a packed (N, sum(sel)) list."""
    offs = np.concatenate([[0], np.cumsum(type_count)]).astype(int)
    cols = np.concatenate([[0], np.cumsum(sel)]).astype(int)
    nt = len(type_count)
    return [[nbrs[offs[i]:offs[i + 1], cols[j]:cols[j + 1]] for j in range(nt)] for i in range(nt)]


def from_nbrs_nm(nbrs_nm, device="cuda"):
    """Packed (N, sum(sel)) int32 list and sel from the reference's nested
    nbrs_nm (type-local indices of the neighbour type, pad N)."""
    rows = []
    for row in nbrs_nm:
        rows.append(torch.cat([torch.as_tensor(np.asarray(a) if not torch.is_tensor(a) else a,
                                               dtype=torch.int32, device=device) for a in row], dim=1))
    sel = [int(np.shape(a)[1]) for a in nbrs_nm[0]]
    return torch.cat(rows, dim=0).contiguous(), sel


@dataclass
class TypedNeighborList:
    """Mirror of deepmd_jax.md_utils.TypedNeighborList (md_utils.py:330-350)."""
    nbrs: torch.Tensor
    knbr: list
    nbrs_nm: list
    did_buffer_overflow: bool
    reference_box: np.ndarray
    status: torch.Tensor = field(default=None, repr=False)

    def set(self, **kw):
        d = dict(self.__dict__)
        d.update(kw)
        return TypedNeighborList(**d)


def typed_neighbor_list(box, type_idx, type_count, rcut, buffer_ratio=1.2):
    """Typed neighbour list functions (deepmd_jax/md_utils.py:353-461).

    ``box`` is the (3,) orthorhombic reference box, ``rcut`` the list cutoff
    (model rcut + skin).  Coordinates passed to allocate/update are (N, 3) in
    the user's atom order; the list refers to the stable type-sorted order.
    """
    _require_cuda()
    type_idx = np.asarray(type_idx, dtype=int)
    type_count = [int(c) for c in type_count]
    ref_box = np.asarray(box, dtype=np.float32).reshape(-1)
    if ref_box.size == 9:
        ref_box = np.diag(ref_box.reshape(3, 3)).copy()
    elif ref_box.size == 1:
        ref_box = np.repeat(ref_box, 3)
    perm, _ = sort_by_type(type_idx, len(type_count))
    perm_dev = torch.tensor(perm.astype(np.int32), device="cuda")
    N = len(type_idx)
    nt = len(type_count)

    def _box3(b):
        if b is None:
            return ref_box
        b = np.asarray(b, dtype=np.float32).reshape(-1)
        if b.size == 9:
            b = np.diag(b.reshape(3, 3)).copy()
        elif b.size == 1:
            b = np.repeat(b, 3)
        return b

    def _coord(coord):
        c = coord if torch.is_tensor(coord) else torch.as_tensor(np.asarray(coord))
        return c.to(device="cuda", dtype=torch.float32).reshape(1, N, 3).contiguous()

    def _cutoff(b):
        return float(rcut * np.max(ref_box / b))

    def _build(coord, b, sel, counts=None):
        nb = NeighborBuilder(N, 1, type_count, sel, b, _cutoff(b), ref_box=ref_box)
        nbrs, status = nb.build(_coord(coord), perm=perm_dev, counts=counts)
        return nbrs[0], status

    def allocate_fn(coord, box=None, knbr_override=None):
        b = _box3(box)
        if knbr_override is None:
            cap = MEASURE_CAPACITY
            while True:
                counts = torch.empty((1, N, nt), dtype=torch.int32, device="cuda")
                _build(coord, b, [cap] * nt, counts=counts)
                mx = counts.reshape(-1, nt).max(0).values.cpu().numpy()
                if mx.max() < cap:
                    break
                cap = int(2 ** np.ceil(np.log2(mx.max() + 2)))
            knbr = knbr_from_counts(mx, buffer_ratio)
            print("# Neighborlist allocated with size %s, rcut_plus_skin = %s, buffer_ratio = %s"
                  % (np.array(knbr) - 1, rcut, buffer_ratio))
        else:
            knbr = [int(k) for k in knbr_override]
        sel = [max(k - 1, 1) for k in knbr]
        nbrs, status = _build(coord, b, sel)
        over = bool(int(status.item()) & 2)
        return TypedNeighborList(nbrs=nbrs, knbr=knbr, nbrs_nm=to_nbrs_nm(nbrs, type_count, sel),
                                 did_buffer_overflow=over, reference_box=ref_box, status=status)

    def update_fn(coord, typed_nbrs, box=None):
        b = _box3(box)
        sel = [max(k - 1, 1) for k in typed_nbrs.knbr]
        nbrs, status = _build(coord, b, sel)
        over = bool(int(status.item()) & 2) or bool(typed_nbrs.did_buffer_overflow)
        return typed_nbrs.set(nbrs=nbrs, nbrs_nm=to_nbrs_nm(nbrs, type_count, sel), did_buffer_overflow=over,
                              status=status)

    return SimpleNamespace(allocate=allocate_fn, update=update_fn)


def exact_neighbor_list(pos, perm, type_count, boxes, rcut):
    """Neighbour lists of F frames at exactly the largest per-type count
    (no overflow possible), for one-shot evaluation where the reference uses
    its lattice path (deepmd_jax/utils.py:54-82, data.py:347-364).

    pos (F, N, 3) float32 CUDA in user order, perm (N,) int32 CUDA
    (type-sorted index -> user index), boxes (F, 3).  Frames that share one
    box are listed in one call.  Returns (nbrs (F, N, sum(sel)), sel)."""
    F, N = int(pos.shape[0]), int(pos.shape[1])
    nt = len(type_count)
    boxes = np.asarray(boxes, dtype=np.float32).reshape(F, 3)
    if (boxes == boxes[0]).all():
        groups = [(0, F)]
    else:
        groups = [(f, f + 1) for f in range(F)]
    cap = MEASURE_CAPACITY
    while True:
        counts = torch.empty((F, N, nt), dtype=torch.int32, device=pos.device)
        for a, b in groups:
            NeighborBuilder(N, b - a, type_count, [cap] * nt, boxes[a], rcut).build(
                pos[a:b], perm=perm, counts=counts[a:b])
        mx = counts.reshape(-1, nt).max(0).values.cpu().numpy()
        if mx.max() < cap:
            break
        cap = int(2 ** np.ceil(np.log2(mx.max() + 2)))
    sel = [max(int(m), 1) for m in mx]
    nbrs = torch.empty((F, N, sum(sel)), dtype=torch.int32, device=pos.device)
    for a, b in groups:
        NeighborBuilder(N, b - a, type_count, sel, boxes[a], rcut).build(pos[a:b], perm=perm, nbrs=nbrs[a:b])
    return nbrs, sel


def min_image_unwrap(previous_position, current_position, box):
    """A step's positions moved by whole box vectors onto the image nearest
    the previous step's (deepmd_jax/md_utils.py:160-167); box (3,) or (3, 3)."""
    prev = np.asarray(previous_position, dtype=np.float64)
    cur = np.asarray(current_position, dtype=np.float64)
    box = np.asarray(box, dtype=np.float64)
    if box.size == 3:
        b = box.reshape(3)
        return prev + np.mod(cur - prev + b / 2, b) - b / 2
    frac = (cur - prev) @ np.linalg.inv(box)
    return prev + (frac - np.round(frac)) @ box


def print_run_profile(steps, elapsed_time, natoms, dt):
    """Per-run timing summary of deepmd_jax/md_utils.py:170-177."""
    steps_per_microsecond_per_atom = 1e-6 * steps * natoms / (elapsed_time + 1e-6)
    nanosecond_per_day = 1e-6 * steps * dt * (86400 / elapsed_time)
    print("# Finished %d steps in %dh %dm %ds." %
          (steps, elapsed_time // 3600, (elapsed_time % 3600) // 60, elapsed_time % 60))
    print("# Performance: %.3f ns/day, %.3f step/μs/atom" %
          (nanosecond_per_day, steps_per_microsecond_per_atom))
