"""General (triclinic) boxes on the CPU: the open ghost-atom system of
lattice.ghost_system holds every periodic image within rcut, and the float64
oracle evaluated on it (ghost rows of the list emptied, the cell atoms'
energies summed, ghost forces folded back) reproduces the reference's own
lattice path on sheared cells (tests/golden/golden_triclinic.npz, from
tests/golden/make_golden_triclinic.py)."""
import os

import numpy as np
import pytest
import torch

from deepmd_jax_b200.lattice import ghost_system
from make_golden import golden_models
from oracle import model as om

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "golden_triclinic.npz"))
RCUT = 6.0


def _image_distances(coord, box, i, rcut, reach=6):
    """Brute force: distances from atom i to every periodic image (other than
    itself) within rcut, over lattice translations up to ``reach``."""
    B = np.asarray(box, float)
    g = np.arange(-reach, reach + 1)
    shifts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) @ B
    d = np.linalg.norm(coord[None, :, :] + shifts[:, None, :] - coord[i], axis=-1)
    d[reach * (2 * reach + 1) ** 2 + reach * (2 * reach + 1) + reach, i] = np.inf  # the atom itself
    return np.sort(d[d < rcut])


@pytest.mark.parametrize("box", [
    np.array([[13.4, 0.0, 0.0], [3.1, 13.0, 0.0], [-2.2, 1.7, 13.2]]),
    np.array([[10.1, 0.0, 0.0], [2.6, 9.8, 0.0], [1.2, -2.1, 9.9]]),
    np.array([[7.0, 0.0, 0.0], [5.5, 6.0, 0.0], [-4.0, 3.5, 6.5]]),   # strongly skewed, narrow
])
def test_ghost_system_holds_every_image_within_rcut(box):
    rng = np.random.default_rng(3)
    coord = rng.uniform(-0.3, 1.3, size=(24, 3)) @ box            # some atoms outside the cell
    pos, src, L = ghost_system(coord, box, RCUT)
    N = len(coord)
    assert (src[:N] == np.arange(N)).all()
    assert (pos.min(0) >= RCUT).all() and (pos.max(0) <= L - RCUT).all()   # no periodic contact in the open box
    for i in range(N):
        want = _image_distances(coord, box, i, RCUT)
        d = np.linalg.norm(pos - pos[i], axis=1)
        d[i] = np.inf
        got = np.sort(d[d < RCUT])
        assert len(got) == len(want), (i, len(got), len(want))
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)


def open_list(pos, src, N, type_idx, ntypes, rcut):
    """Typed list of the open system in the oracle's block layout (type-local
    indices ascending, pad M), ghost rows empty."""
    M = len(pos)
    t = type_idx[src]
    perm, count = om.sort_by_type(t, ntypes)
    ps = pos[perm]
    offs = np.concatenate([[0], np.cumsum(count)])
    d = np.linalg.norm(ps[:, None, :] - ps[None, :, :], axis=-1)
    np.fill_diagonal(d, np.inf)
    hit = d < rcut
    hit[perm >= N] = False                      # ghost centres: no rows
    sel = [max(int(hit[:, offs[j]:offs[j + 1]].sum(1).max()), 1) for j in range(ntypes)]
    nbrs = np.full((M, sum(sel)), M, dtype=np.int64)
    col = np.concatenate([[0], np.cumsum(sel)])
    for j in range(ntypes):
        for r in range(M):
            idx = np.nonzero(hit[r, offs[j]:offs[j + 1]])[0]
            nbrs[r, col[j]:col[j] + len(idx)] = idx
    return nbrs, sel


@pytest.mark.parametrize("name", ["S", "U"])
def test_ghost_system_oracle_matches_reference_lattice_path(name):
    p, v = golden_models()["B"]
    m64 = om.OracleModel(p, v, torch.float64)
    coord, box, types = GOLD[name + "_pos"], GOLD[name + "_box"], GOLD[name + "_type"].astype(int)
    N = len(types)
    pos, src, L = ghost_system(coord, box, RCUT)
    nbrs, sel = open_list(pos, src, N, types, 2, RCUT)
    r = om.energy_force(m64, pos, L, types[src], nbrs=nbrs, sel=sel)
    E = r["atom_energy"][:N].sum()
    F = np.zeros((N, 3))
    np.add.at(F, src, r["force"])
    Eg, Fg = float(GOLD[name + "_E"]), GOLD[name + "_F"]
    assert abs(E - Eg) <= 1e-9 * abs(Eg), (E, Eg)
    np.testing.assert_allclose(F, Fg, rtol=0, atol=1e-9 * np.abs(Fg).max())
