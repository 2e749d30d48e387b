"""Host-side logic of the reference-facing API that needs no GPU: the box
shapes evaluate() accepts and its error message (deepmd_jax/train.py:718-740),
the neighbour capacity rule (deepmd_jax/md_utils.py:394-403), the
conversion between the packed list and the reference's nested nbrs_nm, the
DeepMD data loader and error metrics of test(), periodic_replicate, and the
host arithmetic of the PIMD Invariant and Model_Devi reporters."""
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


@pytest.mark.parametrize("content,n_bead,want", [
    ("positions", 1, ("position",)), ("positions", 3, ("position", "centroid")),
    ("all", 1, ("position", "velocity")), ("all", 2, ("position", "velocity", "centroid")),
    (["velocity", "position"], 1, ("position", "velocity")), (("centroid", "all"), 2, ("position", "velocity", "centroid")),
    (iter(["velocity"]), 1, ("velocity",)), ("velocity", 1, ("velocity",)),
])
def test_dump_content_vocabulary(content, n_bead, want):
    """dump_content words and kinds (deepmd_jax/md_utils.py:30-68): file
    order position, velocity, centroid whatever the request order."""
    from deepmd_jax_b200 import dump
    assert dump.normalize_content(content, n_bead) == want


@pytest.mark.parametrize("content,msg", [
    ([], "must not be empty"), ([1, "position"], "entries must be strings"), (5, "or an iterable"),
    (["pos"], r"Unknown dump_content entries \['pos'\]"), ("centroid", "only meaningful when n_bead > 1"),
])
def test_dump_content_errors(content, msg):
    from deepmd_jax_b200 import dump
    with pytest.raises(ValueError, match=msg):
        dump.normalize_content(content, 1)


def _write_dp_dir(root, type_idx, sets):
    """A DeepMD-format directory: type.raw and set.NNN/{coord,box,energy,force}.npy."""
    root.mkdir(parents=True, exist_ok=True)
    (root / "type.raw").write_text("\n".join(str(int(t)) for t in type_idx))
    for k, frames in enumerate(sets):
        d = root / ("set.%03d" % k)
        d.mkdir()
        for name, arr in frames.items():
            np.save(d / (name + ".npy"), arr.reshape(arr.shape[0], -1) if arr.ndim > 1 else arr)


def test_dp_loader_and_error_metrics(tmp_path):
    """test()'s data side (deepmd_jax/data.py:190-200, train.py:629-690):
    two directories (two compositions), sets concatenated in sorted order,
    and the metric formulas checked on hand-made predictions."""
    from deepmd_jax_b200.train import error_metrics, load_dp_data
    rng = np.random.default_rng(0)

    def frames(nf, n):
        return {"coord": rng.normal(size=(nf, n, 3)), "box": np.tile(np.eye(3) * 9.0, (nf, 1, 1)),
                "energy": rng.normal(size=nf), "force": rng.normal(size=(nf, n, 3))}
    a_sets = [frames(2, 5), frames(3, 5)]
    b_sets = [frames(1, 4)]
    _write_dp_dir(tmp_path / "a", [0, 1, 1, 0, 1], a_sets)
    _write_dp_dir(tmp_path / "b", [1, 0, 0, 1], b_sets)
    leaves = load_dp_data([str(tmp_path / "a"), [str(tmp_path / "b")]])
    assert [len(l["energy"]) for l in leaves] == [5, 1]
    assert np.array_equal(leaves[0]["type_idx"], [0, 1, 1, 0, 1])
    assert np.allclose(leaves[0]["coord"], np.concatenate([s["coord"] for s in a_sets]))
    assert leaves[0]["box"].shape == (5, 3, 3) and leaves[1]["force"].shape == (1, 4, 3)
    with pytest.raises(NotImplementedError):
        load_dp_data(str(tmp_path / "x.extxyz"))

    results, dE, dF = [], [], []
    for leaf in leaves:
        for i in range(len(leaf["energy"])):
            pe = leaf["energy"][i] + rng.normal()
            pf = leaf["force"][i] + rng.normal(size=leaf["force"][i].shape)
            results.append({"type_idx": leaf["type_idx"], "predicted_energy": pe, "true_energy": leaf["energy"][i],
                            "predicted_force": pf, "true_force": leaf["force"][i]})
            dE.append((pe - leaf["energy"][i]) / len(leaf["type_idx"]))
            dF.append(pf - leaf["force"][i])
    m = error_metrics(results)
    dE = np.array(dE)
    allF = np.concatenate([d.reshape(-1) for d in dF])
    per_atom = np.concatenate([np.sqrt((d ** 2).mean(-1)) for d in dF])
    assert np.isclose(m["rmse"]["energy"], np.sqrt((dE ** 2).mean()))
    assert np.isclose(m["mae"]["energy"], np.abs(dE).mean()) and np.isclose(m["l1_mixed"]["energy"], np.abs(dE).mean())
    assert np.isclose(m["rmse"]["force"], np.sqrt((allF ** 2).mean()))
    assert np.isclose(m["mae"]["force"], np.abs(allF).mean())
    assert np.isclose(m["l1_mixed"]["force"], per_atom.mean())


def test_periodic_replicate():
    """utils.periodic_replicate (deepmd_jax/utils.py:299-327): copies along
    x, then y, then z, each axis's copies outermost; scalar, (3,) and (3, 3)
    boxes; tiled types, forces and velocities."""
    from deepmd_jax_b200.utils import periodic_replicate
    rng = np.random.default_rng(1)
    c = rng.uniform(0, 3, size=(4, 3))
    t = np.array([0, 1, 1, 0])
    f = rng.normal(size=(4, 3))
    out = periodic_replicate([2, 1, 3], c, [3.0, 4.0, 5.0], type_idx=t, force=f, velocity=f * 2)
    assert np.array_equal(out[1], [6.0, 4.0, 15.0])
    want = np.array([c[a] + np.array([ix * 3.0, 0.0, iz * 5.0])
                     for iz in range(3) for ix in range(2) for a in range(4)])
    assert np.allclose(out[0], want)
    assert np.array_equal(out[2], np.tile(t, 6)) and np.array_equal(out[3], np.concatenate([f] * 6))
    assert np.array_equal(out[4], np.concatenate([2 * f] * 6))
    c2, b2 = periodic_replicate(2, c, 3.0)
    assert np.array_equal(b2, [6.0, 6.0, 6.0]) and c2.shape == (32, 3)
    c3, b3 = periodic_replicate(2, c, np.diag([3.0, 4.0, 5.0]))
    assert np.array_equal(b3, np.diag([6.0, 8.0, 10.0]))
    assert np.allclose(c3[-1], c[-1] + [3.0, 4.0, 5.0])


def _stub_simulation(**attrs):
    """A Simulation object without an engine: only the attributes the
    report helpers read (no GPU)."""
    from deepmd_jax_b200.md import Simulation
    sim = Simulation.__new__(Simulation)
    for k, v in attrs.items():
        setattr(sim, k, v)
    return sim


def test_pimd_invariant_formula_on_host():
    """The ring-polymer Invariant of md.py:512-557 as the host computes it
    from the engine's report and bead positions: NVT and NPT forms against
    an independent evaluation with the oracle's unwrap across beads."""
    import types
    from oracle import integrators as oi
    from deepmd_jax_b200.md import PRESS_UNIT_CONVERSION
    rng = np.random.default_rng(2)
    P, N = 4, 6
    box = np.array([7.0, 8.0, 9.0])
    R = rng.uniform(0, 1, size=(P, N, 3)) * box + rng.integers(-1, 2, size=(P, N, 3)) * box
    mass = rng.uniform(1, 16, size=N)
    kT = 300.0 * 8.617333e-5
    rep = types.SimpleNamespace(kinetic_energy=1.7, potential_energy=-40.2, thermostat_work=0.3,
                                box=tuple(box * 1.01), ngroups=2, box_momentum=(0.2, -0.1, 0.0),
                                box_mass=(50.0, 70.0, 1.0), box_thermostat_work=0.05)
    m = (mass * 103.6427)[:, None]
    omega = P * kT / oi.HBAR
    for routine, bx in (("NVT", box), ("NPT", box * 1.01)):
        sim = _stub_simulation(_n_bead=P, _routine=routine, _box=box, _mass=mass, _kT=kT, _pressure=2.0,
                               getPosition=lambda: R)
        Ru = oi.unwrap_across_beads(R, bx)
        spring = 0.5 * omega ** 2 * float((m * (Ru - np.roll(Ru, 1, axis=0)) ** 2).sum())
        want = (1.7 - 40.2 + spring - 0.3) / P
        if routine == "NPT":
            want += 0.5 * 0.2 ** 2 / 50.0 + 0.5 * 0.1 ** 2 / 70.0 + 2.0 * PRESS_UNIT_CONVERSION * np.prod(bx) - 0.05
        assert np.isclose(sim._pimd_invariant(rep), want, rtol=1e-12, atol=1e-12)


def test_model_deviation_is_max_std_over_models():
    """Model_Devi (md.py:559-567): max over atoms and axes of the standard
    deviation (ddof 0) over the deviation models' forces."""
    rng = np.random.default_rng(4)
    F = rng.normal(size=(3, 5, 3))
    sim = _stub_simulation(_dev_models=[object()] * 3, _deviation_forces=lambda: F)
    assert sim.model_deviation() == pytest.approx(float(np.max(np.std(F, axis=0))))
    with pytest.raises(ValueError):
        _stub_simulation(_dev_models=[]).model_deviation()


@pytest.mark.parametrize("axes,gid", [(((0, 1, 2),), [0, 0, 0]), (((0, 1),), [0, 0, -1]), (((0,),), [0, -1, -1]),
                                      (((0,), (1,), (2,)), [0, 1, 2]), (((0, 1), (2,)), [0, 0, 1])])
def test_couple_axes_groups(axes, gid):
    """couple_axes (deepmd_jax/routine.py:199-229): the documented examples
    map each axis to its group, -1 for a fixed axis."""
    from deepmd_jax_b200.md import parse_couple_axes
    groups, got = parse_couple_axes(axes)
    assert groups == axes and got == gid


@pytest.mark.parametrize("bad,msg", [((0, 1), "tuple of tuples"), (((0, 3),), "must be in"),
                                     (((0, 1), (1,)), "partition"), (((0,), ()), "non-empty"),
                                     ((), "at least one group")])
def test_couple_axes_errors(bad, msg):
    from deepmd_jax_b200.md import parse_couple_axes
    with pytest.raises(ValueError, match=msg):
        parse_couple_axes(bad)


def test_trajectory_helpers_match_oracle():
    """Host post-processing helpers with the reference's names: bead unwrap,
    centroid and spring energy (deepmd_jax/pimd.py:82-89,210-248) against the
    oracle's, and min_image_unwrap (md_utils.py:160-167) for (3,) and
    diagonal (3, 3) boxes."""
    from oracle import integrators as oi
    from deepmd_jax_b200 import pimd
    from deepmd_jax_b200.md_utils import min_image_unwrap
    rng = np.random.default_rng(9)
    box = np.array([5.0, 6.0, 7.0])
    R = rng.uniform(0, 1, size=(4, 5, 3)) * box + rng.integers(-2, 3, size=(4, 5, 3)) * box
    assert np.allclose(pimd.unwrap_across_beads(R, box), oi.unwrap_across_beads(R, box), atol=1e-12)
    assert np.allclose(pimd.unwrap_across_beads(R, np.diag(box)), oi.unwrap_across_beads(R, box), atol=1e-12)
    assert np.allclose(pimd.centroid(R, box), oi.unwrap_across_beads(R, box).mean(0), atol=1e-12)
    sim = _stub_simulation(_box=box)  # the centroid frames Simulation.run returns under PIMD
    assert np.allclose(sim._centroid(R), pimd.centroid(R, box)) and np.allclose(sim._centroid(R, box * 2),
                                                                                 pimd.centroid(R, box * 2))
    m = rng.uniform(1, 10, size=(5, 1))
    Ru = oi.unwrap_across_beads(R, box)
    want = 0.5 * 0.3 ** 2 * float((m * (Ru - np.roll(Ru, 1, axis=0)) ** 2).sum())
    assert np.isclose(pimd.spring_energy(R, m, box, 0.3), want, rtol=1e-12)
    prev = rng.uniform(0, 1, size=(5, 3)) * box
    cur = prev + rng.normal(scale=0.1, size=(5, 3)) + rng.integers(-1, 2, size=(5, 3)) * box
    want = oi.min_image_unwrap(prev, cur, box)
    assert np.allclose(min_image_unwrap(prev, cur, box), want, atol=1e-12)
    assert np.allclose(min_image_unwrap(prev, cur, np.diag(box)), want, atol=1e-12)


@pytest.mark.parametrize("kw,exc,msg", [
    (dict(routine="NVT", pimd_lambda=-1.0), ValueError, "pimd_lambda must be non-negative"),
    (dict(routine="NVE", n_bead=2), NotImplementedError, "currently supports routine='NVT' or 'NPT'"),
    (dict(routine="NVT", n_bead=2, fixed_indices=[0]), NotImplementedError, "fixed_indices is not supported"),
    (dict(routine="NVT", n_bead=2, model_deviation_paths=["m.pkl"]), NotImplementedError,
     "model_deviation_paths is not supported"),
    (dict(routine="NVT", n_bead=2, remove_com_motion=True), NotImplementedError, "remove_com_motion is not"),
    (dict(routine="NVT", couple_axes=((0, 1),)), ValueError, "couple_axes is only meaningful"),
    (dict(routine="NVT_berendsen"), NotImplementedError, "routine currently limited"),
    (dict(routine="NPT", fixed_indices=[0], pressure=1.0), NotImplementedError, "Fixing atoms currently limited"),
    (dict(routine="NPT"), ValueError, "Missing argument 'pressure'"),
    (dict(routine="NPT", pressure=1.0, couple_axes=((0, 0),)), ValueError, "partition"),
])
def test_simulation_argument_errors_before_device_work(kw, exc, msg):
    """Simulation's argument checks run before any device work and raise what
    the reference raises (deepmd_jax/md.py:136-165,242-244,228-229,324,
    382-383), so they hold on a machine without a GPU."""
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import init_dp_params, water_box
    p, v = init_dp_params(seed=0)
    w = water_box(2, 6.21, seed=0)
    args = dict(temperature=300.0)
    args.update(kw)
    routine = args.pop("routine")
    with pytest.raises(exc, match=msg):
        Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], routine, 0.5, w["position"], **args)


def test_simulation_rejects_unknown_atomic_numbers():
    """type_idx holds atomic numbers when the model carries chemical_types;
    unknown ones raise the reference's ValueError (md.py:176-181)."""
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import init_dp_params, water_box
    p, v = init_dp_params(seed=0)
    p = dict(p, chemical_types=(8, 1))
    w = water_box(2, 6.21, seed=0)
    z = np.where(w["type_idx"] == 0, 8, 6)
    with pytest.raises(ValueError, match="not in model.params"):
        Simulation((p, v), w["box"], z, w["mass_per_type"], "NVE", 0.5, w["position"])


def test_set_position_argument_errors():
    """setPosition's checks (deepmd_jax/md.py:989-1006) on a stub engine:
    wrong shape, a box outside NPT, a box of another shape or an
    anisotropic change under NPT."""
    sim = _stub_simulation(_is_pimd=False, _routine="NVT", _natoms=3, _n_bead=1,
                           getBox=lambda: np.array([5.0, 5.0, 6.0]))
    sim._frame_shape = lambda: (3, 3)
    with pytest.raises(ValueError, match="same shape as the initial position"):
        sim.setPosition(np.zeros((4, 3)))
    with pytest.raises(ValueError, match="only be changed in NPT"):
        sim.setPosition(np.zeros((3, 3)), box=5.0)
    sim._routine = "NPT"
    with pytest.raises(ValueError, match="same shape as the initial box"):
        sim.setPosition(np.zeros((3, 3)), box=np.eye(3))
    with pytest.raises(ValueError, match="isotropic"):
        sim.setPosition(np.zeros((3, 3)), box=[5.0, 5.5, 6.0])


class _FakeEngineLib:
    """The dpb_md_* calls run() makes between chunks, as no-ops returning 0."""

    def __init__(self):
        self.restores = 0

    def dpb_md_snapshot(self, h, restore):
        self.restores += int(restore)
        return 0

    def dpb_md_clear_status(self, h, mask):
        return 0


def _scripted_run(codes, steps=30, chunk=10):
    """Simulation.run on a stub engine whose chunk status words come from
    `codes` in turn; each recorded chunk writes its call number into the
    trajectory rows it covers."""
    import types
    import torch
    N = 2
    calls = []
    sim = _stub_simulation(
        _type_idx=np.zeros(N, dtype=int), _type_symbols=None, _n_bead=1, report_interval=chunk,
        _step_chunk_size=chunk, _is_initial_state=False, _box=np.array([5.0, 5.0, 5.0]), _natoms=N,
        _routine="NVE", _is_pimd=False, verbose=False, _dt=0.5, step=0, _buffer_ratio=1.2, _h=None,
        _traj_bufs=[(torch.zeros(chunk, N * 3), torch.zeros(chunk, N * 3)) for _ in range(2)])
    sim.lib = _FakeEngineLib()
    sim._frame_shape = lambda: (N, 3)
    script = list(codes)
    reports, resized = [], []

    def run_chunk(n, p, v):
        calls.append(n)

    def copy_out(pending, traj):
        _, _, n, idx, tag = pending
        traj["position"][idx:idx + n] = tag

    sim._run_chunk = run_chunk
    sim._report_struct = lambda: types.SimpleNamespace(status=script.pop(0) if script else 0)
    sim._chunk_event = lambda: len(calls)
    sim._copy_out = copy_out
    sim._report_row = lambda tic: reports.append(sim.step)
    sim._resize_capacity = lambda: resized.append(sim.step)
    traj = sim.run(steps)
    return sim, traj, calls, reports, resized


def test_run_records_nan_chunk_then_stops():
    """Status bit 16 (NaN/Inf) as the reference handles it (deepmd_jax/md.py:
    906-950): the chunk is still committed - its frames recorded, the step
    advanced, the report printed - and the run ends there."""
    sim, traj, calls, reports, _ = _scripted_run([0, 16])
    assert calls == [10, 10] and sim.step == 20 and reports == [10, 20]
    assert np.all(traj["position"][:10] == 1) and np.all(traj["position"][10:20] == 2)
    assert np.all(traj["position"][20:] == 0) and sim._error_code == 16


@pytest.mark.parametrize("codes,restores", [([18], 1), ([2, 16], 2)])
def test_run_discards_nan_chunk_with_overflow(codes, restores):
    """NaN together with a hard overflow (error word not 0, 4 or 16), or right
    after a neighbour reallocation (word 20): the reference resolves the
    error and leaves without recording that chunk (md.py:906-916)."""
    sim, traj, calls, reports, resized = _scripted_run(codes)
    assert sim.step == 0 and reports == [] and np.all(traj["position"] == 0)
    assert sim.lib.restores == restores and len(calls) == len(codes)
    assert resized == [0]  # one reallocation, at step 0, in both scripts


def _reference_style_pickle(params, variables):
    """A model.pkl byte stream as the reference writes it (deepmd_jax/utils.py:
    225-228) on a machine with jax and flax: the DPModel flax Module pickles as
    its class deepmd_jax.dpmodel.DPModel plus its instance dict (params,
    parent, name, flax's _ModuleInternalState with a SetupState member), the
    variables tree as nested FrozenDicts, each leaf a jax.Array reduced to
    jax._src.array._reconstruct_array(numpy reconstructor, args, ndarray
    state, {'weak_type': False}).  Neither jax nor flax is installed here, so
    the globals are served by stand-in modules registered under those names
    only while pickling."""
    import enum
    import pickle
    import sys
    import types
    names = ["deepmd_jax", "deepmd_jax.dpmodel", "jax", "jax._src", "jax._src.array", "flax", "flax.core",
             "flax.core.frozen_dict", "flax.linen", "flax.linen.module"]
    saved = {n: sys.modules.get(n) for n in names}
    mods = {n: types.ModuleType(n) for n in names}

    def _reconstruct_array(fun, args, arr_state, aval_state):  # never called while pickling
        raise AssertionError

    _reconstruct_array.__module__, _reconstruct_array.__qualname__ = "jax._src.array", "_reconstruct_array"
    mods["jax._src.array"]._reconstruct_array = _reconstruct_array

    class ArrayImpl:
        def __init__(self, a):
            self.a = np.asarray(a)

        def __reduce__(self):
            fun, args, arr_state = self.a.__reduce__()
            return _reconstruct_array, (fun, args, arr_state, {"weak_type": False})

    class FrozenDict(dict):
        def __reduce__(self):
            return FrozenDict, (dict(self),)

    FrozenDict.__module__, FrozenDict.__qualname__ = "flax.core.frozen_dict", "FrozenDict"
    mods["flax.core.frozen_dict"].FrozenDict = FrozenDict
    SetupState = enum.IntEnum("SetupState", [("NEW", 0), ("TRANSFORMED", 1), ("DONE", 2)],
                              module="flax.linen.module")
    mods["flax.linen.module"].SetupState = SetupState

    class _ModuleInternalState:
        pass

    _ModuleInternalState.__module__ = "flax.linen.module"
    _ModuleInternalState.__qualname__ = "_ModuleInternalState"
    mods["flax.linen.module"]._ModuleInternalState = _ModuleInternalState

    class DPModel:
        pass

    DPModel.__module__, DPModel.__qualname__ = "deepmd_jax.dpmodel", "DPModel"
    mods["deepmd_jax.dpmodel"].DPModel = DPModel

    def tree(x):
        if isinstance(x, dict):
            return FrozenDict({k: tree(v) for k, v in x.items()})
        return ArrayImpl(x)

    try:
        sys.modules.update(mods)
        st = _ModuleInternalState()
        st.__dict__.update(in_compact_method=False, in_setup=False, setup_called=SetupState.NEW,
                           is_initialized=False, autoname_cursor={}, children={})
        model = DPModel()
        model.__dict__.update(params=params, parent=None, name=None, _state=st)
        return pickle.dumps({"model": model, "variables": tree(variables)}, protocol=4)
    finally:
        for n, m in saved.items():
            if m is None:
                sys.modules.pop(n, None)
            else:
                sys.modules[n] = m


def test_load_model_reads_reference_pickle_globals(tmp_path):
    """load_model on a stream that names the real jax / flax globals: the
    globals are exactly the allow-listed ones, the parameters and every
    variable leaf come back as the writer's numpy values."""
    import io
    from deepmd_jax_b200 import utils
    from deepmd_jax_b200.systems import init_dp_params
    from deepmd_jax_b200.utils import load_model
    p, v = init_dp_params(seed=3)
    blob = _reference_style_pickle(p, v)
    globs = set()

    class Recorder(utils._Unpickler):
        def find_class(self, module, name):
            globs.add((module, name))
            return super().find_class(module, name)

    Recorder(io.BytesIO(blob)).load()
    assert {("deepmd_jax.dpmodel", "DPModel"), ("jax._src.array", "_reconstruct_array"),
            ("flax.core.frozen_dict", "FrozenDict"), ("flax.linen.module", "_ModuleInternalState"),
            ("flax.linen.module", "SetupState")} <= globs
    path = tmp_path / "model.pkl"
    path.write_bytes(blob)
    model, variables = load_model(str(path))
    assert model.params["embed_widths"] == p["embed_widths"] and model.params["rcut"] == p["rcut"]

    def leaves(t, pre=""):
        for k, x in t.items():
            if isinstance(x, dict):
                yield from leaves(x, pre + k + "/")
            else:
                yield pre + k, x

    got, want = dict(leaves(variables)), dict(leaves(v))
    assert got.keys() == want.keys()
    for k in want:
        assert isinstance(got[k], np.ndarray) and got[k].dtype == np.asarray(want[k]).dtype
        assert np.array_equal(got[k], want[k]), k


def test_load_model_refuses_unknown_globals(tmp_path):
    """A global outside the allow-list fails loudly instead of loading as a
    stand-in."""
    import pickle
    import collections
    from deepmd_jax_b200.utils import load_model
    path = tmp_path / "bad.pkl"
    path.write_bytes(pickle.dumps({"model": collections.Counter(), "variables": {}}))
    with pytest.raises(pickle.UnpicklingError, match="collections.Counter"):
        load_model(str(path))


@pytest.mark.parametrize("n_side,L", [(4, 12.42), (8, 24.83), (16, 49.66)])
def test_no_pair_within_an_ulp_of_the_cutoff(n_side, L):
    """jax_md's float32 summation order of d^2 is unpinned (oracle/nlist.py);
    the neighbour sets cannot depend on it when no pair's float32 d^2 lies
    within one ulp of (rcut + skin)^2.  Checked on the initial frames of the
    192-, 1,536- and 12,288-atom water boxes (rcut 6 A, skin 0.3 A)."""
    from oracle import nlist as onl
    from deepmd_jax_b200.systems import water_box
    w = water_box(n_side, L, seed=0)
    c = onl.canonicalize(w["position"], w["box"], w["type_idx"])
    assert onl.boundary_pairs(c, w["box"].astype(np.float32), onl.cutoff_sq(6.3)) == 0


def test_serving_latency_split_and_batch_phases():
    """Server.latency_summary splits each request's latency into queue time
    (submit -> taken into a batch or MD slot) and service time, and
    batch_summary averages the host phases of the evaluation batches; the
    HBM budget admits first come first served and never exceeds its total.
    Host logic only (a stand-in for the server's state, no device)."""
    import threading
    import types
    from deepmd_jax_b200.serving import HBMBudget, Server, _Req
    reqs = []
    for k, (kind, q, s) in enumerate([("eval", 0.01, 0.05), ("eval", 0.02, 0.03), ("eval", 0.03, 0.01),
                                      ("md", 0.5, 1.0)]):
        r = _Req(kind, None, 0, 10, 1)
        r.t_submit, r.t_start, r.t_done = 100.0 + k, 100.0 + k + q, 100.0 + k + q + s
        reqs.append(r)
    stub = types.SimpleNamespace(completed=reqs, _lock=threading.Condition(),
                                 batch_log=[{"requests": 2, "atoms": 100, "pack_s": 0.001, "launch_s": 0.002,
                                             "wait_s": 0.004, "handout_s": 0.0005},
                                            {"requests": 4, "atoms": 300, "pack_s": 0.003, "launch_s": 0.004,
                                             "wait_s": 0.002, "handout_s": 0.0015}])
    lat = Server.latency_summary(stub)
    assert lat["eval"]["n"] == 3 and lat["md"]["n"] == 1
    assert lat["eval"]["p50_s"] == pytest.approx(0.05)
    assert lat["eval"]["queue_p50_s"] == pytest.approx(0.02)
    assert lat["eval"]["service_p50_s"] == pytest.approx(0.03)
    assert lat["md"]["queue_p50_s"] == pytest.approx(0.5) and lat["md"]["service_p50_s"] == pytest.approx(1.0)
    ph = Server.batch_summary(stub)
    assert ph["batches"] == 2 and ph["mean_requests"] == 3.0 and ph["mean_atom_frames"] == 200.0
    assert ph["pack_s"]["mean"] == pytest.approx(0.002) and ph["wait_s"]["max"] == pytest.approx(0.004)
    b = HBMBudget(100)
    assert b.try_reserve(60) and not b.try_reserve(50) and b.try_reserve(40)
    b.release(60)
    assert b.try_reserve(50) and b.peak == 100 and b.used == 90


def test_serving_request_boxes():
    """The serving loop's box shapes: one box (3,) or (3, 3) for every frame,
    per-frame boxes in evaluate()'s shapes; general boxes and bad shapes
    rejected before anything is queued."""
    from deepmd_jax_b200.serving import request_boxes
    t = np.zeros(5, dtype=int)
    c2, c3 = np.zeros((2, 5, 3), np.float32), np.zeros((3, 5, 3), np.float32)
    L = np.array([10.0, 11.0, 12.5])
    assert np.array_equal(request_boxes(L, c2, t), np.stack([L, L]).astype(np.float32))
    assert np.array_equal(request_boxes(np.diag(L), c2, t), np.stack([L, L]).astype(np.float32))
    per = np.array([[10.0, 11.0, 12.0], [13.0, 14.0, 15.0]])
    assert np.array_equal(request_boxes(per, c2, t), per.astype(np.float32))
    assert np.array_equal(request_boxes(np.stack([np.diag(b) for b in per]), c2, t), per.astype(np.float32))
    assert np.array_equal(request_boxes(np.array([9.0, 8.0]), c2, t), np.array([[9.0] * 3, [8.0] * 3], np.float32))
    assert np.array_equal(request_boxes(np.stack([np.diag(b).reshape(9) for b in per]), c2, t),
                          per.astype(np.float32))
    # a (3, 3) array with three frames is three rows of lengths, as evaluate() reads it
    rows = np.array([[10.0, 10.0, 10.0], [11.0, 11.0, 11.0], [12.0, 12.0, 12.0]])
    assert np.array_equal(request_boxes(rows, c3, t), rows.astype(np.float32))
    sheared = np.diag(L)
    sheared[1, 0] = 2.0
    with pytest.raises(NotImplementedError, match="orthorhombic"):
        request_boxes(sheared, c2, t)
    with pytest.raises(ValueError):
        request_boxes(np.ones((4, 3)), c2, t)
