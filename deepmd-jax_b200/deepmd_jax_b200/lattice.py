"""General (triclinic) periodic boxes on the evaluation path.

The reference evaluates frames on its lattice path: each pair displacement
is moved into the parallelepiped around the origin (``shift`` with
``ortho=False``, deepmd_jax/utils.py:20-27) and offset by the lattice
candidates of ``compute_lattice_candidate`` (deepmd_jax/data.py:347-364,
utils.py:66-78), so every periodic image within rcut of an atom contributes.

The device kernels take the orthorhombic minimum image, so a frame in a
general box is turned into an open (non-periodic) system with the same
energy first: the atoms, wrapped into the cell, plus "ghost" copies at the
lattice translations whose fractional coordinates lie within
rcut |b*_k| of the cell on every axis (b*_k the k-th reciprocal vector;
1 / |b*_k| is the spacing of the lattice planes), which holds every image
within rcut of any point of the cell.  The ghosts' own rows of the
neighbour list are emptied, so only the cell's atoms are centres: the energy
is the sum of their atomic energies, the force on a ghost is added to the
atom it copies, and the virial summed over the pairs of the cell's centres is
the periodic virial.  The open system sits in an orthorhombic box wider than
its extent plus 2 rcut + 2 A on every axis, so no pair meets a periodic image
there.  Unlike the reference, whose candidate search is a heuristic that can
miss images in strongly skewed cells (data.py:348), every image within rcut
is found.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import sort_by_type


def is_orthorhombic(box):
    """True for a (3, 3) box without off-diagonal entries."""
    b = np.asarray(box, dtype=np.float64).reshape(3, 3)
    return not np.any(b - np.diag(np.diag(b)))


def ghost_system(coord, box, rcut):
    """Open system of one frame in a general box.

    coord (N, 3), box (3, 3) with the lattice vectors as rows (coord = frac @
    box, the reference's convention).  Returns (pos (M, 3) float64 inside the
    open box, src (M,) int64: the cell atom each of the M atoms copies, the
    first N being the atoms themselves, L (3,) float64: the open box)."""
    B = np.asarray(box, dtype=np.float64).reshape(3, 3)
    x = np.asarray(coord, dtype=np.float64).reshape(-1, 3)
    N = x.shape[0]
    if abs(np.linalg.det(B)) < 1e-12:
        raise ValueError("box is singular")
    inv = np.linalg.inv(B)
    frac = x @ inv
    frac -= np.floor(frac)
    frac[frac >= 1.0] = 0.0
    delta = rcut * np.linalg.norm(inv, axis=0) + 1e-9   # rcut |b*_k| per axis
    reach = np.ceil(delta).astype(int)
    fr, src = [frac], [np.arange(N)]
    for a in range(-reach[0], reach[0] + 1):
        for b in range(-reach[1], reach[1] + 1):
            for c in range(-reach[2], reach[2] + 1):
                if a == 0 and b == 0 and c == 0:
                    continue
                f = frac + np.array([a, b, c], dtype=np.float64)
                keep = np.all((f >= -delta) & (f < 1.0 + delta), axis=1)
                if keep.any():
                    fr.append(f[keep])
                    src.append(np.nonzero(keep)[0])
    pos = np.concatenate(fr) @ B
    src = np.concatenate(src).astype(np.int64)
    lo, hi = pos.min(0), pos.max(0)
    margin = rcut + 1.0
    L = (hi - lo) + 2.0 * margin
    return pos - lo + margin, src, L


def ghost_eval(dm, coord, box, type_idx, ntypes, rcut, precision, virial=False, descriptors=False):
    """Energy, forces (N, 3) float32 in the input order and, with ``virial``,
    the 3x3 virial W = -sum_ij r_ij (x) f_ij of one frame in a general box
    (the open system of ``ghost_system``), on the device model ``dm``.  With
    ``descriptors`` also the descriptor T of the cell's atoms in their
    type-sorted order (the reference's debug output)."""
    from .md_utils import exact_neighbor_list
    type_idx = np.asarray(type_idx, dtype=int)
    N = len(type_idx)
    pos, src, L = ghost_system(coord, box, rcut)
    M = len(src)
    tix = type_idx[src]
    perm, count = sort_by_type(tix, ntypes)
    perm_dev = torch.tensor(perm.astype(np.int32), device="cuda")
    p = torch.tensor(pos[None].astype(np.float32), device="cuda")
    nbrs, sel = exact_neighbor_list(p, perm_dev, count, L[None], rcut)
    ghost_rows = torch.tensor(np.nonzero(perm >= N)[0], dtype=torch.int64, device="cuda")
    if ghost_rows.numel():
        nbrs[0, ghost_rows] = M                           # ghosts are neighbours, never centres
    bx = torch.tensor(L[None].astype(np.float32), device="cuda")
    out = dm.evaluate(p, bx, nbrs, count, sel, perm=perm_dev, atom_energy=True, precision=precision)
    st = int(out["status"].item())
    if st & 16:
        raise FloatingPointError("NaN/Inf in the evaluation (status %d)" % st)
    ea = out["atom_energy"][0, :N].double().cpu().numpy()
    f_ext = out["force"][0].double().cpu().numpy()
    force = np.zeros((N, 3), dtype=np.float64)
    np.add.at(force, src, f_ext)
    res = {"energy": float(ea.sum()), "force": force.astype(np.float32)}
    if virial:
        res["virial"] = out["virial"][0].cpu().numpy().reshape(3, 3)
    if descriptors:
        T, _ = dm.descriptors(p, bx, nbrs, count, sel, perm=perm_dev, precision=precision)
        # the stable type sort puts each type's cell atoms (indices < N) first in its block
        offs = np.concatenate([[0], np.cumsum(count)])
        n_cell = np.bincount(type_idx, minlength=ntypes)
        rows = np.concatenate([np.arange(offs[t], offs[t] + n_cell[t]) for t in range(ntypes)])
        res["T"] = T[torch.as_tensor(rows, device=T.device)].cpu().numpy()
    return res
