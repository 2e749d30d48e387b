"""Host-side logic of the reference-facing API that needs no GPU: the box
shapes evaluate() accepts and its error message (deepmd_jax/train.py:718-740),
the neighbour capacity rule (deepmd_jax/md_utils.py:394-403) and the
conversion between the packed list and the reference's nested nbrs_nm."""
import numpy as np
import pytest
import torch

from oracle import nlist as onl


def test_box_shapes_of_evaluate():
    from deepmd_jax_b200.train import normalize_boxes
    F, N = 2, 6
    coord = np.zeros((F, N, 3))
    t = np.zeros(N, dtype=int)
    want = np.stack([np.diag([5.0, 5.0, 5.0])] * F)
    for b in (np.full(F, 5.0), np.full((F, 1), 5.0), np.full((F, 3), 5.0), want.reshape(F, 9), want):
        assert np.array_equal(normalize_boxes(coord, b, t), want)
    for bad_coord, bad_box, bad_t in ((coord[0], np.full(F, 5.0), t), (coord, np.full(F + 1, 5.0), t),
                                      (coord, np.full(F, 5.0), t[:-1]), (coord, np.zeros((F, 3, 2)), t)):
        with pytest.raises(ValueError, match="Input shapes are incorrect"):
            normalize_boxes(bad_coord, bad_box, bad_t)


def test_non_orthorhombic_box_is_rejected():
    from deepmd_jax_b200.dpmodel import box_diagonal
    assert np.array_equal(box_diagonal(4.0), [4.0, 4.0, 4.0])
    assert np.array_equal(box_diagonal(np.diag([1.0, 2.0, 3.0])), [1.0, 2.0, 3.0])
    tri = np.diag([5.0, 5.0, 5.0])
    tri[0, 1] = 1.0
    with pytest.raises(NotImplementedError):
        box_diagonal(tri)


@pytest.mark.parametrize("ratio", [1.2, 1.25, 1.5])
def test_capacity_rule_matches_oracle(ratio):
    from deepmd_jax_b200.md_utils import knbr_from_counts
    from deepmd_jax_b200.md import sel_from_counts
    for counts in ([0, 5], [19, 20], [46, 92], [1, 300]):
        want = [int(k) for k in onl.knbr_rule(counts, ratio)]
        assert knbr_from_counts(counts, ratio) == want
        assert sel_from_counts(counts, ratio) == [max(k - 1, 1) for k in want]


def test_nested_and_packed_lists_round_trip():
    from deepmd_jax_b200.md_utils import from_nbrs_nm, to_nbrs_nm
    cnt, sel = [3, 5], [2, 4]
    rng = np.random.default_rng(0)
    packed = torch.tensor(rng.integers(0, 9, size=(8, 6)), dtype=torch.int32)
    nested = to_nbrs_nm(packed, cnt, sel)
    assert [tuple(a.shape) for a in nested[0]] == [(3, 2), (3, 4)]
    assert [tuple(a.shape) for a in nested[1]] == [(5, 2), (5, 4)]
    back, sel2 = from_nbrs_nm([[a.numpy() for a in row] for row in nested], device="cpu")
    assert sel2 == sel and torch.equal(back, packed)


def test_packed_batch_layout():
    """Layout of the serving loop's packed batches: slots are a bijection,
    each frame's type runs start at multiples of 8, padding atoms carry
    -(s+1), and every real atom's slot holds its own type."""
    from deepmd_jax_b200.engine import PackedBatch
    rng = np.random.default_rng(0)
    items = [(rng.integers(0, 2, 13), 2, [5.0, 5.0, 5.0]), (rng.integers(0, 2, 30), 1, [7.0, 7.0, 7.0]),
             (np.array([1, 1, 1]), 3, [4.0, 4.0, 4.0])]
    b = PackedBatch(items, 2)
    assert sorted(b.perm.tolist()) == list(range(b.natoms))
    assert b.nseg == 6 and b.nreal == 13 * 2 + 30 + 3 * 3
    slot_type = np.full(b.natoms, -1)
    for (t, nf, _), it in zip(items, b.items):
        for f in range(nf):
            slot_type[it["slot0"] + f * len(t):it["slot0"] + (f + 1) * len(t)] = t
    offs = np.concatenate([[0], np.cumsum(b.type_count)])
    for k in range(b.natoms):
        ty = int(np.searchsorted(offs, k, side="right") - 1)
        if b.seg[k] >= 0:
            assert slot_type[b.perm[k]] == ty
        else:
            assert b.perm[k] >= b.nreal
    for it in b.items:
        for t in range(2):
            assert it["stride"][t] % 8 == 0 and it["base0"][t] % 8 == 0
            for f in range(it["nframes"]):
                rows = it["row0"][t] + f * it["stride"][t] + np.arange(it["stride"][t])
                n = int(it["type_count"][t])
                assert np.all(b.seg[rows[:n]] == it["seg0"] + f)
                assert np.all(b.seg[rows[n:]] == -(it["seg0"] + f) - 1)


def test_xyz_dump_format_and_options(tmp_path):
    """Trajectory dump files (deepmd_jax/md_utils.py:30-256): names, option
    errors and the extended-XYZ frame text."""
    from deepmd_jax_b200 import dump
    prefix = str(tmp_path / "traj")
    with pytest.raises(ValueError, match="type_symbols"):
        dump.prepare([0, 1], None, 1, 10, dump_prefix=prefix)
    with pytest.raises(ValueError, match="centroid"):
        dump.prepare([0, 1], ["O", "H"], 1, 10, dump_prefix=prefix, dump_content=["centroid"])
    with pytest.raises(ValueError, match="requires dump_prefix"):
        dump.prepare([0, 1], ["O", "H"], 1, 10, dump_content=["velocity"])
    assert dump.normalize_content("positions", 4) == ("position", "centroid")
    assert dump.normalize_content("all", 1) == ("position", "velocity")
    d, k = dump.prepare([0, 1, 1], ["O", "H"], 1, 10, dump_interval=5, dump_prefix=prefix, dump_content="all")
    assert k == 5 and [x[1] for x in d] == [prefix + "_position.xyz", prefix + "_velocity.xyz"]
    pos = np.array([[1.0, 2.0, 3.0], [0.5, 0.25, 0.125], [4.0, 5.0, 6.0]])
    dump.write_frame(d, pos, 2 * pos, None, [12.42, 12.42, 12.42], step=5)
    text = open(prefix + "_position.xyz").read().splitlines()
    assert text[0] == "3"
    assert text[1] == ('Lattice="12.42000000 0.00000000 0.00000000 0.00000000 12.42000000 0.00000000 0.00000000 '
                       '0.00000000 12.42000000" Properties=species:S:1:pos:R:3 step=5 pbc="T T T"')
    assert text[2] == "O  1.00000000 2.00000000 3.00000000"
    frames = dump.read_xyz(prefix + "_velocity.xyz")
    assert frames[0][0] == ["O", "H", "H"] and np.allclose(frames[0][1], 2 * pos)
    d2, _ = dump.prepare([0, 1, 1], ["O", "H"], 2, 10, dump_prefix=prefix)
    assert [x[1] for x in d2] == [prefix + "_position_bead0.xyz", prefix + "_position_bead1.xyz",
                                  prefix + "_centroid.xyz"]
