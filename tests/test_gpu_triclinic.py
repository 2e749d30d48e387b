"""General (triclinic) boxes on the GPU through the open ghost-atom system
(lattice.ghost_eval): evaluate(), DPModel and the ASE calculator against the
reference's own lattice path (golden_triclinic.npz, from the unmodified
reference source) and against the float64 oracle on the same open system.

Bars as for orthorhombic boxes: FP32 energy within 2e-6 sum|E_atom| + 1e-6
eV, forces within 2e-4 of max|F|, virial within 2e-4 of max|W|; mixed form
force RMS error <= 5e-3 eV/A and <= 3e-2 of the force RMS, energy per atom
within 2e-2 of mean |E_atom|."""
import os

import numpy as np
import pytest
import torch

from make_golden import golden_models
from oracle import model as om
from test_gpu_api import _Atoms
from test_triclinic_cpu import GOLD, RCUT, open_list

pytestmark = pytest.mark.gpu

MODELS = golden_models()
_ORACLE = {}


def _oracle(name):
    """float64 oracle on the open system of golden frame ``name``: energy,
    per-atom energies of the cell atoms, folded forces, virial."""
    if name not in _ORACLE:
        from deepmd_jax_b200.lattice import ghost_system
        coord, box, types = GOLD[name + "_pos"], GOLD[name + "_box"], GOLD[name + "_type"].astype(int)
        N = len(types)
        pos, src, L = ghost_system(coord, box, RCUT)
        nbrs, sel = open_list(pos, src, N, types, 2, RCUT)
        r = om.energy_force(om.OracleModel(*MODELS["B"], torch.float64), pos, L, types[src], nbrs=nbrs, sel=sel)
        F = np.zeros((N, 3))
        np.add.at(F, src, r["force"])
        _ORACLE[name] = dict(E=r["atom_energy"][:N].sum(), Ea=r["atom_energy"][:N], F=F, W=r["virial"])
    return _ORACLE[name]


def _pkl(tmp_path):
    from deepmd_jax_b200.utils import save_model
    path = str(tmp_path / "model_B.pkl")
    save_model(path, *MODELS["B"])
    return path


def _check(E, F, name, prec):
    Eg, Fg, Ea = float(GOLD[name + "_E"]), GOLD[name + "_F"], _oracle(name)["Ea"]
    if prec == "fp32":
        assert abs(E - Eg) <= 2e-6 * np.abs(Ea).sum() + 1e-6, (E, Eg)
        assert np.abs(F - Fg).max() <= 2e-4 * np.abs(Fg).max(), (np.abs(F - Fg).max(), np.abs(Fg).max())
    else:
        rms = np.sqrt(((F - Fg) ** 2).mean())
        assert rms <= 5e-3 and rms <= 3e-2 * np.sqrt((Fg ** 2).mean()), rms
        assert abs(E - Eg) / len(Ea) <= 2e-2 * np.abs(Ea).mean(), (E, Eg)


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
@pytest.mark.parametrize("name", ["S", "U"])
def test_evaluate_general_box_matches_reference_lattice_path(tmp_path, name, prec):
    from deepmd_jax_b200.train import evaluate
    coord, box, types = GOLD[name + "_pos"], GOLD[name + "_box"], GOLD[name + "_type"]
    out = evaluate(_pkl(tmp_path), coord[None], box[None], types, precision=prec)
    _check(out["energy"][0], out["force"][0], name, prec)
    if prec == "fp32":   # the oracle on the open system agrees with the reference's lattice path
        o = _oracle(name)
        assert abs(o["E"] - float(GOLD[name + "_E"])) <= 1e-9 * abs(o["E"])


def test_evaluate_mixes_orthorhombic_and_general_frames(tmp_path):
    """One call with frames in orthorhombic and general boxes (batch_size 2):
    each frame's energy and forces as when evaluated alone; a lattice
    translation of a frame changes nothing."""
    from deepmd_jax_b200.train import evaluate
    G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_model.npz"))
    A_pos, A_box, A_type = G["A_pos"], G["A_box"], G["A_type"]
    S_pos, S_box, S_type = GOLD["S_pos"], GOLD["S_box"], GOLD["S_type"]
    assert (A_type == S_type).all()
    coord = np.stack([A_pos, S_pos, A_pos + 0.37, S_pos + S_box[1] - S_box[2]])
    boxes = np.stack([np.diag(A_box), S_box, np.diag(A_box), S_box])
    out = evaluate(_pkl(tmp_path), coord, boxes, A_type, batch_size=2)
    EB, FB = float(G["B_E"]), G["B_F"]
    for f in (0, 2):
        assert abs(out["energy"][f] - EB) <= 2e-6 * abs(EB) + 1e-6
        assert np.abs(out["force"][f] - FB).max() <= 2e-4 * np.abs(FB).max()
    for f in (1, 3):
        _check(out["energy"][f], out["force"][f], "S", "fp32")


def test_dpmodel_virial_and_ase_stress_general_box(tmp_path):
    """DPModel.energy_force_virial and DPJaxCalculator on the sheared 192-atom
    cell: virial against the float64 oracle on the open system, stress
    -W / |det cell| in Voigt order; a typed neighbour list with a general box
    is rejected (the reference's list path reads only the box diagonal)."""
    from deepmd_jax_b200.ase_calc import DPJaxCalculator
    from deepmd_jax_b200.dpmodel import DPModel
    p, v = MODELS["B"]
    coord, box, types = GOLD["S_pos"], GOLD["S_box"], GOLD["S_type"].astype(int)
    E, F, W = DPModel(p).energy_force_virial(v, coord, box, {"type_idx": tuple(types)})
    _check(E, F, "S", "fp32")
    Wo = _oracle("S")["W"]
    assert np.abs(W - Wo).max() <= 2e-4 * np.abs(Wo).max(), (W, Wo)
    calc = DPJaxCalculator(_pkl(tmp_path), type_idx=types)
    atoms = _Atoms(coord, box)
    S = calc.get_stress(atoms)
    ref = -np.array([Wo[0, 0], Wo[1, 1], Wo[2, 2], Wo[1, 2], Wo[0, 2], Wo[0, 1]]) / abs(np.linalg.det(box))
    assert np.abs(S - ref).max() <= 2e-4 * np.abs(ref).max()
    with pytest.raises(NotImplementedError):
        DPModel(p).energy(v, coord, box, {"type_idx": tuple(types)}, nbrs_nm=[[np.zeros((64, 1), int)] * 2] * 2)
