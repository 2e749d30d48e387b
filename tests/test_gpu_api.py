"""The reference-facing API on the GPU: evaluate() (deepmd_jax/train.py:703),
DPModel.apply / energy_and_force (deepmd_jax/dpmodel.py:10-108) and
typed_neighbor_list (deepmd_jax/md_utils.py:353-461), checked against the
golden vectors of the reference model source and against the float64 oracle.

Tolerances are those of the FP32 kernels against FP64 (test_gpu_eval.py):
energy |dE| <= 2e-6 * |E| + 1e-6 eV (the per-atom energies of these models
share one sign, so |E| = sum|E_atom|), forces max|dF| <= 2e-4 * max|F|.
"""
import os

import numpy as np
import pytest
import torch

from make_golden import golden_models
from oracle import model as om
from oracle import nlist as onl

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_model.npz"))
MODELS = golden_models()


def _close(E, F, E_ref, F_ref, N):
    assert abs(E - E_ref) <= 2e-6 * abs(E_ref) + 1e-6, (E, E_ref, N)
    fmax = np.abs(F_ref).max()
    assert np.abs(F - F_ref).max() <= 2e-4 * fmax, (np.abs(F - F_ref).max(), fmax)


def _pkl(tmp_path, key):
    from deepmd_jax_b200.utils import save_model
    p, v = MODELS[key]
    path = str(tmp_path / ("model_%s.pkl" % key))
    save_model(path, p, v)
    return path


def test_evaluate_frames_and_box_shapes_match_reference(tmp_path):
    from deepmd_jax_b200.train import evaluate
    path = _pkl(tmp_path, "A")
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    rng = np.random.default_rng(7)
    coord = np.stack([pos, pos + rng.normal(scale=0.05, size=pos.shape), pos + 0.37])
    m = om.OracleModel(*MODELS["A"], torch.float64)
    ref1 = om.energy_force(m, coord[1], box, typ, virial=False)
    for bshape in ("scalar", "diag", "matrix"):
        b = {"scalar": np.full(3, box[0]), "diag": np.stack([box] * 3),
             "matrix": np.stack([np.diag(box)] * 3)}[bshape]
        out = evaluate(path, coord, b, typ, batch_size=2)
        assert out["energy"].shape == (3,) and out["force"].shape == (3, 192, 3)
        _close(out["energy"][0], out["force"][0], float(G["A_E"]), G["A_F"], 192)
        _close(out["energy"][1], out["force"][1], ref1["energy"], ref1["force"], 192)
        # a rigid translation changes nothing
        _close(out["energy"][2], out["force"][2], float(G["A_E"]), G["A_F"], 192)


def test_evaluate_small_box_sums_images_like_reference_lattice_path(tmp_path):
    from deepmd_jax_b200.train import evaluate
    path = _pkl(tmp_path, "B")
    pos, box, typ = G["E_pos"], G["E_box"], G["E_type"]
    out = evaluate(path, pos[None], box[None], typ)
    _close(out["energy"][0], out["force"][0], float(G["E_E"]), G["E_F"], len(typ))


def test_evaluate_unsorted_types_and_chemical_types(tmp_path):
    """Atoms in an arbitrary order, given as atomic numbers (O=8, H=1)."""
    from deepmd_jax_b200.train import evaluate
    from deepmd_jax_b200.utils import save_model
    p, v = MODELS["B"]
    p = dict(p)
    p["chemical_types"] = (8, 1)                 # type 0 is Z=8, type 1 is Z=1
    path = str(tmp_path / "model_z.pkl")
    save_model(path, p, v)
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    order = np.random.default_rng(1).permutation(len(typ))
    z = np.where(typ[order] == 0, 8, 1)
    out = evaluate(path, pos[order][None], box[None], z)
    _close(out["energy"][0], out["force"][0], float(G["B_E"]), G["B_F"][order], 192)
    with pytest.raises(ValueError):
        evaluate(path, pos[None], box[None], np.full(192, 6))


def test_dpmodel_apply_with_and_without_typed_list():
    from deepmd_jax_b200.dpmodel import DPModel
    from deepmd_jax_b200.md_utils import typed_neighbor_list
    p, v = MODELS["B"]
    pos, box, typ = G["D_pos"], G["D_box"], G["D_type"]
    cnt = np.bincount(typ, minlength=2)
    model = DPModel(p)
    fns = typed_neighbor_list(box, typ, cnt, 6.3)
    nb = fns.allocate(pos)
    assert not nb.did_buffer_overflow
    # the capacity rule of allocate_fn
    c = onl.canonicalize(pos, box, typ)
    _, counts, _ = onl.typed_nlist(c, box.astype(np.float32), onl.cutoff_sq(6.3), cnt, [256, 256])
    assert nb.knbr == [int(k) for k in onl.knbr_rule(counts.reshape(-1, 2).max(0))]
    E1, F1 = model.energy_and_force(v, pos, np.diag(box), {"type_idx": tuple(typ)}, nb.nbrs_nm)
    E2, F2 = model.energy_and_force(v, pos, np.diag(box), {"type_idx": tuple(typ)})
    _close(E1, F1, float(G["D_E"]), G["D_F"], len(typ))
    _close(E2, F2, float(G["D_E"]), G["D_F"], len(typ))
    # nbrs_nm handed back in the reference's nested form gives the same result
    nested = [[a.cpu().numpy() for a in row] for row in nb.nbrs_nm]
    E3, F3 = model.energy_and_force(v, pos, box, {"type_idx": tuple(typ)}, nested)
    # (force sums use float atomics, so the last bit may differ between calls)
    assert abs(E3 - E1) <= 1e-9 * abs(E1) and np.abs(F3 - F1).max() <= 1e-6 * np.abs(F1).max()
    # update after a small move keeps the capacity and the sets
    pos2 = pos + np.random.default_rng(2).normal(scale=0.05, size=pos.shape)
    nb2 = fns.update(pos2, nb)
    assert nb2.knbr == nb.knbr and not nb2.did_buffer_overflow
    E4, F4 = model.energy_and_force(v, pos2, box, {"type_idx": tuple(typ)}, nb2.nbrs_nm)
    c2 = onl.canonicalize(pos2, box, typ)
    typed2, _, _ = onl.typed_nlist(c2, box.astype(np.float32), onl.cutoff_sq(6.3), cnt, [64, 128])
    ref = om.energy_force(om.OracleModel(p, v, torch.float64), pos2, box, typ, nbrs=typed2, sel=[64, 128],
                          virial=False)
    _close(E4, F4, ref["energy"], ref["force"], len(typ))


def test_typed_list_sets_match_oracle_exactly():
    from deepmd_jax_b200.md_utils import typed_neighbor_list
    pos, box, typ = G["D_pos"], G["D_box"], G["D_type"]
    cnt = np.bincount(typ, minlength=2)
    nb = typed_neighbor_list(box, typ, cnt, 6.3).allocate(pos, knbr_override=[47, 93])
    got = nb.nbrs.cpu().numpy()
    assert np.array_equal(got, G["D_nbrs"])
    assert [tuple(a.shape) for a in nb.nbrs_nm[0]] == [(cnt[0], 46), (cnt[0], 92)]
    assert [tuple(a.shape) for a in nb.nbrs_nm[1]] == [(cnt[1], 46), (cnt[1], 92)]


def test_adjoint_matches_central_differences():
    """Force from the hand-written adjoint vs central differences of the
    device energy (h = 1e-3 A, 64 random atom components) and of the FP64
    oracle energy.  The device energy is an FP64 sum of FP32 per-atom
    energies; a 1e-3 A move changes only the atoms within rcut of the moved
    one; the float32 per-atom energies of those ~100 atoms carry ~1e-6
    relative rounding (1600-wide dot products), so the device difference
    quotient is noisy at ~1e-6 eV / 2e-3 A ~ 5e-4 eV/A: its bar is 1e-2 of
    the largest force, the float64 one 2e-3."""
    from deepmd_jax_b200.dpmodel import DPModel, EnergyFunction
    p, v = MODELS["B"]
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    model = DPModel(p)
    sa = {"type_idx": tuple(typ)}
    E0, F0 = model.energy_and_force(v, pos, box, sa)
    m64 = om.OracleModel(p, v, torch.float64)
    rng = np.random.default_rng(11)
    comps = [(int(a), int(k)) for a, k in zip(rng.integers(0, len(typ), 64), rng.integers(0, 3, 64))]
    h = 1e-3
    fd_dev, fd_64 = [], []
    for a, k in comps:
        dp = np.zeros_like(pos)
        dp[a, k] = h
        fd_dev.append(-(model.energy(v, pos + dp, box, sa) - model.energy(v, pos - dp, box, sa)) / (2 * h))
        fd_64.append(-(om.energy_only(m64, pos + dp, box, typ)[0] - om.energy_only(m64, pos - dp, box, typ)[0]) / (2 * h))
    f_adj = np.array([F0[a, k] for a, k in comps])
    fd_dev, fd_64 = np.array(fd_dev), np.array(fd_64)
    scale = np.abs(F0).max()
    assert np.abs(f_adj - fd_64).max() <= 2e-3 * scale, np.abs(f_adj - fd_64).max()
    assert np.abs(f_adj - fd_dev).max() <= 1e-2 * scale, np.abs(f_adj - fd_dev).max()
    # torch autograd through the adjoint node
    x = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    e = EnergyFunction.apply(x, model, v, box, typ)
    e.backward()
    assert np.allclose(-x.grad.numpy(), F0, rtol=0, atol=1e-6)


def test_evaluate_compressed_model_pkl(tmp_path):
    """A model.pkl carrying compress_var (the default output of the
    reference's train(), deepmd_jax/train.py:31) evaluates through the
    compressed tables: against the float64 oracle with the same tables."""
    from deepmd_jax_b200.train import evaluate
    from deepmd_jax_b200.utils import save_model
    from make_golden import hermite_compressed
    p, v = hermite_compressed(*MODELS["B"])
    path = str(tmp_path / "model_cmp.pkl")
    save_model(path, p, v)
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    out = evaluate(path, pos[None], box[None], typ)
    ref = om.energy_force(om.OracleModel(p, v, torch.float64), pos, box, typ, virial=False)
    _close(out["energy"][0], out["force"][0], ref["energy"], ref["force"], len(typ))


class _Atoms:
    """The part of ase.Atoms the calculator reads (ASE is not installed)."""

    def __init__(self, positions, cell):
        self._p, self._c = np.array(positions, float), np.array(cell, float)

    def copy(self):
        return _Atoms(self._p, self._c)

    def get_positions(self):
        return self._p.copy()

    def get_cell(self, complete=False):
        return self._c.copy()


def test_ase_calculator_energy_forces_stress(tmp_path):
    """DPJaxCalculator (deepmd_jax/ase_calc.py:18-144): energy and forces of
    the reference golden vectors; stress = -W / V in Voigt order against the
    float64 oracle's virial."""
    from deepmd_jax_b200.ase_calc import DPJaxCalculator
    path = _pkl(tmp_path, "B")
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    calc = DPJaxCalculator(path, type_idx=typ)
    atoms = _Atoms(pos, np.diag(box))
    E, F, S = calc.get_potential_energy(atoms), calc.get_forces(atoms), calc.get_stress(atoms)
    _close(E, F, float(G["B_E"]), G["B_F"], len(typ))
    W = om.energy_force(om.OracleModel(*MODELS["B"], torch.float64), pos, box, typ)["virial"]
    V = float(np.prod(box))
    ref = -np.array([W[0, 0], W[1, 1], W[2, 2], W[1, 2], W[0, 2], W[0, 1]]) / V
    assert S.shape == (6,) and np.abs(S - ref).max() <= 2e-4 * np.abs(ref).max() + 1e-12


def test_test_on_dp_directories_matches_golden_and_metrics(tmp_path):
    """test() (deepmd_jax/train.py:523-701) on three DeepMD-format
    directories (the 192-, 1,536- and 96-atom golden systems of model B, two
    sets each, the second set a rigid translation), labels = golden values
    plus known offsets: predictions match the golden vectors and the
    metrics are those of the offsets."""
    from deepmd_jax_b200.train import test as dp_test
    path = _pkl(tmp_path, "B")
    rng = np.random.default_rng(3)
    expect = []
    dirs = []
    for sysk, key in (("A", "B"), ("D", "D"), ("E", "E")):
        pos, box, typ = G[sysk + "_pos"], G[sysk + "_box"], G[sysk + "_type"]
        root = tmp_path / ("data_" + sysk)
        (root).mkdir()
        (root / "type.raw").write_text("\n".join(str(int(t)) for t in typ))
        for k, shift in enumerate((0.0, 0.41)):
            d = root / ("set.%03d" % k)
            d.mkdir()
            dE = rng.normal()
            dF = rng.normal(scale=0.1, size=pos.shape)
            np.save(d / "coord.npy", (pos + shift).reshape(1, -1))
            np.save(d / "box.npy", np.diag(box).reshape(1, 9))
            np.save(d / "energy.npy", np.array([float(G[key + "_E"]) + dE]))
            np.save(d / "force.npy", (G[key + "_F"] + dF).reshape(1, -1))
            expect.append((float(G[key + "_E"]), G[key + "_F"], dE, dF, len(typ)))
        dirs.append(str(root))
    metrics, results = dp_test(path, dirs, batch_size=2)
    assert len(results) == 6
    e_err, f_err = [], []
    for r, (E, F, dE, dF, n) in zip(results, expect):
        _close(r["predicted_energy"], r["predicted_force"], E, F, n)
        assert np.isclose(r["true_energy"], E + dE) and r["box"].shape == (3, 3)
        e_err.append((r["predicted_energy"] - r["true_energy"]) / n)
        f_err.append((r["predicted_force"] - r["true_force"]).reshape(-1))
    e_err, f_err = np.array(e_err), np.concatenate(f_err)
    assert np.isclose(metrics["rmse"]["energy"], np.sqrt((e_err ** 2).mean()))
    assert np.isclose(metrics["rmse"]["force"], np.sqrt((f_err ** 2).mean()), rtol=1e-5)
    # the metrics are those of the planted offsets to the FP32 error
    assert abs(metrics["rmse"]["energy"] - np.sqrt(np.mean([(x[2] / x[4]) ** 2 for x in expect]))) < 1e-4


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_apply_debug_descriptor_matches_oracle(precision):
    """DPModel.apply returns (energy, T_NselXW) like the reference
    (deepmd_jax/dpmodel.py:50-51,99-100): T (N, 10, W) / Nnbrs without Tbias,
    type-sorted, against the FP64 oracle's T - to 1e-5 of max |T| in FP32,
    to 2e-2 RMS (relative) in the mixed form (FP16 embedding operands)."""
    from deepmd_jax_b200.dpmodel import DPModel
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["B"]
    w = water_box(4, 12.42, seed=0)
    e, T = DPModel(p, precision=precision).apply(v, w["position"], w["box"], {"type_idx": tuple(w["type_idx"])})
    _, _, T_ref = om.energy_only(om.OracleModel(p, v, torch.float64), w["position"], w["box"], w["type_idx"])
    T_ref = T_ref.numpy()
    assert T.shape == T_ref.shape == (192, 10, p["embed_widths"][-1])
    if precision == "fp32":
        assert np.abs(T - T_ref).max() <= 1e-5 * np.abs(T_ref).max()
    else:
        assert np.sqrt(((T - T_ref) ** 2).mean()) <= 2e-2 * np.sqrt((T_ref ** 2).mean())
