"""Neighbour list on the GPU vs the brute-force oracle: bit-exact typed
index sets (reference nbrs_nm semantics)."""
import numpy as np
import pytest
import torch

from deepmd_jax_b200.systems import water_box
from oracle import nlist as onl

pytestmark = pytest.mark.gpu


def gpu_nlist(w, sel, rc, perm_input=False, ref_box=None, nframes=1, positions=None):
    from deepmd_jax_b200.engine import NeighborBuilder, sort_by_type
    perm, cnt = sort_by_type(w["type_idx"], 2)
    pos = w["position"] if positions is None else positions
    if perm_input:
        p = torch.tensor(np.ascontiguousarray(pos), dtype=torch.float32, device="cuda").reshape(nframes, -1, 3)
        pm = torch.tensor(perm, dtype=torch.int32, device="cuda")
    else:
        p = torch.tensor(np.ascontiguousarray(np.asarray(pos).reshape(nframes, -1, 3)[:, perm]),
                         dtype=torch.float32, device="cuda")
        pm = None
    nb = NeighborBuilder(len(perm), nframes, cnt, sel, w["box"], rc, ref_box=ref_box)
    counts = torch.empty((nframes, len(perm), 2), dtype=torch.int32, device="cuda")
    ref_pos = torch.empty((nframes, len(perm), 3), dtype=torch.float32, device="cuda")
    nbrs, status = nb.build(p, perm=pm, counts=counts, ref_pos=ref_pos)
    torch.cuda.synchronize()
    return nbrs.cpu().numpy(), counts.cpu().numpy(), int(status.item()), ref_pos.cpu().numpy(), cnt


@pytest.mark.parametrize("n_side,L,seed", [(8, 24.83, 0), (8, 24.83, 7), (16, 49.66, 1)])
@pytest.mark.parametrize("perm_input", [False, True])
def test_nlist_bit_exact(n_side, L, seed, perm_input):
    w = water_box(n_side, L, seed=seed)
    sel = [46, 92]
    got, counts, status, ref_pos, cnt = gpu_nlist(w, sel, 6.3, perm_input=perm_input)
    c = onl.canonicalize(w["position"], w["box"], w["type_idx"])
    assert np.array_equal(ref_pos[0], c)
    want, wcounts, ovf = onl.typed_nlist(c, w["box"].astype(np.float32), onl.cutoff_sq(6.3), cnt, sel)
    assert np.array_equal(got[0], want)
    assert np.array_equal(counts[0], wcounts)
    assert (status & 2 != 0) == ovf


def test_nlist_overflow_flag_and_prefix():
    w = water_box(8, 24.83, seed=2)
    sel = [20, 40]
    got, counts, status, _, cnt = gpu_nlist(w, sel, 6.3)
    c = onl.canonicalize(w["position"], w["box"], w["type_idx"])
    want, wcounts, ovf = onl.typed_nlist(c, w["box"].astype(np.float32), onl.cutoff_sq(6.3), cnt, sel)
    assert ovf and (status & 2)
    assert np.array_equal(got[0], want)


def test_nlist_scaled_reference_box():
    """Box differs from the reference box: coordinates are scaled into the
    reference frame and the cutoff grows by max(ref/box) (md_utils.py:364-410)."""
    w = water_box(8, 24.83, seed=4)
    box = w["box"] * 0.99
    ref_box = w["box"]
    w2 = dict(w, box=box)
    got, counts, status, _, cnt = gpu_nlist(w2, [46, 92], 6.3, ref_box=ref_box)
    c = onl.canonicalize(w["position"], box, w["type_idx"], ref_box=ref_box)
    want, _, _ = onl.typed_nlist(c, ref_box.astype(np.float32), onl.cutoff_sq(6.3, ref_box, box), cnt, [46, 92])
    assert np.array_equal(got[0], want)


def test_nlist_frames_batch():
    ws = [water_box(8, 24.83, seed=s) for s in range(3)]
    pos = np.stack([w["position"] for w in ws])
    got, counts, status, _, cnt = gpu_nlist(ws[0], [46, 92], 6.3, nframes=3, positions=pos)
    for f, w in enumerate(ws):
        c = onl.canonicalize(w["position"], w["box"], w["type_idx"])
        want, _, _ = onl.typed_nlist(c, w["box"].astype(np.float32), onl.cutoff_sq(6.3), cnt, [46, 92])
        assert np.array_equal(got[f], want)


def test_nlist_full_size_sampled_rows_bit_exact():
    """The 98,304-atom box of the MD benchmark (32,768 waters, L = 99.3 A):
    300 sampled centre rows (and the first and last atom of each type block)
    bit-exact against the oracle's float32 distance test over all atoms, and
    on every row the size-independent layout: each type block ascending,
    then padded with N."""
    w = water_box(32, 99.3, seed=3)
    sel = [46, 92]
    got, counts, status, ref_pos, cnt = gpu_nlist(w, sel, 6.3)
    assert (status & 2 != 0) == bool((counts[0] > np.asarray(sel)[None, :]).any())
    c = onl.canonicalize(w["position"], w["box"], w["type_idx"])
    assert np.array_equal(ref_pos[0], c)
    N = len(c)
    rng = np.random.default_rng(0)
    rows = np.unique(np.concatenate([rng.choice(N, 300, replace=False), [0, cnt[0] - 1, cnt[0], N - 1]]))
    L = w["box"].astype(np.float32)
    rc2 = onl.cutoff_sq(6.3)
    offs = np.concatenate([[0], np.cumsum(cnt)])
    col = np.concatenate([[0], np.cumsum(sel)])
    for i in rows:
        d2 = onl.pair_d2(c[i][None, :], c, L)
        m = d2 < rc2
        m[i] = False
        s = np.nonzero(m)[0]
        for j in range(2):
            nb = s[(s >= offs[j]) & (s < offs[j + 1])] - offs[j]
            assert counts[0][i, j] == len(nb)
            want = np.full(sel[j], N, dtype=np.int32)  # pad N (md_utils.py:444-452)
            k = min(len(nb), sel[j])
            want[:k] = nb[:k]
            assert np.array_equal(got[0][i, col[j]:col[j + 1]], want), (i, j)
    for j in range(2):
        blk = got[0][:, col[j]:col[j + 1]].astype(np.int64)
        valid = blk < cnt[j]
        assert (valid | (blk == N)).all()
        assert np.array_equal(valid.sum(1), np.minimum(counts[0][:, j], sel[j]))
        assert (valid[:, :-1] | ~valid[:, 1:]).all()           # pads only after the neighbours
        d = np.diff(blk, axis=1)
        assert ((d > 0) | ~valid[:, 1:]).all()                  # strictly ascending neighbours
