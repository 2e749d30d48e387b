"""FP32 evaluation on the GPU vs the float64 oracle and vs the golden
vectors produced from the reference's own model source.

Tolerances (FP32 kernels against FP64): energy |dE| <= 2e-6 * sum|E_atom| +
1e-6 eV; forces max|dF| <= 2e-4 * max|F|; virial max|dW| <= 2e-4 * max|W|.
"""
import os

import numpy as np
import pytest
import torch

from gpu_helpers import run_gpu
from make_golden import golden_models
from oracle import model as om

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_model.npz"))
MODELS = golden_models()


def check_close(got, ref, name):
    eabs = np.abs(ref["atom_energy"]).sum()
    assert abs(got["energy"] - ref["energy"]) <= 2e-6 * eabs + 1e-6, (name, got["energy"], ref["energy"])
    fmax = np.abs(ref["force"]).max()
    assert np.abs(got["force"] - ref["force"]).max() <= 2e-4 * fmax, (name, np.abs(got["force"] - ref["force"]).max(), fmax)
    if ref.get("virial") is not None:
        wmax = np.abs(ref["virial"]).max()
        assert np.abs(got["virial"] - ref["virial"]).max() <= 2e-4 * wmax + 1e-9, name
    if ref.get("atom_energy") is not None:
        assert np.abs(got["atom_energy"] - ref["atom_energy"]).max() <= 2e-6 * np.abs(ref["atom_energy"]).max() + 1e-6


@pytest.mark.parametrize("key,sysk,mk", [("A", "A", "A"), ("B", "A", "B"), ("D", "D", "B"), ("E", "E", "B")])
def test_fp32_vs_reference_golden(key, sysk, mk):
    p, v = MODELS[mk]
    pos, box, typ = G[sysk + "_pos"], G[sysk + "_box"], G[sysk + "_type"]
    got = run_gpu(p, v, pos, box, typ)
    assert got["status"] == 0
    ref_o = om.energy_force(om.OracleModel(p, v, torch.float64), pos, box, typ)
    ref = dict(energy=float(G[key + "_E"]), force=G[key + "_F"], atom_energy=ref_o["atom_energy"],
               virial=ref_o["virial"])
    check_close(dict(energy=got["energy"][0], force=got["force"][0], virial=got["virial"][0],
                     atom_energy=got["atom_energy"][0]), ref, key)


def test_fp32_batched_frames_match_single():
    from deepmd_jax_b200.systems import water_box
    p, v = MODELS["B"]
    ws = [water_box(8, 24.83, seed=s) for s in (11, 12, 13)]
    pos = np.stack([w["position"] for w in ws])
    got = run_gpu(p, v, pos, ws[0]["box"], ws[0]["type_idx"])
    m = om.OracleModel(p, v, torch.float64)
    for f, w in enumerate(ws):
        ref = om.energy_force(m, w["position"], w["box"], w["type_idx"],
                              nbrs=got["nbrs"][f], sel=[46, 92])
        check_close(dict(energy=got["energy"][f], force=got["force"][f], virial=got["virial"][f],
                         atom_energy=got["atom_energy"][f]), ref, "frame%d" % f)


def test_fp32_default_train_widths():
    """The reference train() default architecture (embed 32-32-64, fit
    128^3, axis 12; deepmd_jax/train.py:24-27)."""
    from deepmd_jax_b200.systems import water_box, init_dp_params
    from make_golden import randomize_model
    w = water_box(8, 24.83, seed=5)
    p, v = randomize_model(*init_dp_params(embed_widths=(32, 32, 64), fit_widths=(128, 128, 128), axis=12,
                                           nnbrs=90.0, seed=3), seed=4)
    got = run_gpu(p, v, w["position"], w["box"], w["type_idx"])
    ref = om.energy_force(om.OracleModel(p, v, torch.float64), w["position"], w["box"], w["type_idx"],
                          nbrs=got["nbrs"][0], sel=[46, 92])
    check_close(dict(energy=got["energy"][0], force=got["force"][0], virial=got["virial"][0],
                     atom_energy=got["atom_energy"][0]), ref, "default")


def test_nonfinite_sets_status_bit():
    p, v = MODELS["B"]
    pos = G["A_pos"].copy()
    pos[3, 0] = np.nan
    got = run_gpu(p, v, pos, G["A_box"], G["A_type"])
    assert got["status"] & 16


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_compressed_model_neighbour_list_path(precision):
    """Compressed embedding tables (deepmd_jax/utils.py:126-151) on a 1,536-atom
    box through the neighbour list, two frames; FP32 at the FP32 bars, mixed
    (FP32 tables + BF16 fitting) at the mixed bars.  The tables are C2
    piecewise quintics fitted to model B the way compress_model builds them;
    the golden model C (random, discontinuous tables) pins only the float64
    oracle, because a float32 lookup can land in the neighbouring interval
    of a discontinuous table."""
    from deepmd_jax_b200.systems import water_box
    from make_golden import hermite_compressed
    p, v = hermite_compressed(*MODELS["B"])
    ws = [water_box(8, 24.83, seed=s) for s in (21, 22)]
    pos = np.stack([w["position"] for w in ws])
    got = run_gpu(p, v, pos, ws[0]["box"], ws[0]["type_idx"], precision=precision)
    assert got["status"] == 0
    m = om.OracleModel(p, v, torch.float64)
    for f, w in enumerate(ws):
        ref = om.energy_force(m, w["position"], w["box"], w["type_idx"], nbrs=got["nbrs"][f], sel=[46, 92])
        one = dict(energy=got["energy"][f], force=got["force"][f], virial=got["virial"][f],
                   atom_energy=got["atom_energy"][f])
        if precision == "fp32":
            check_close(one, ref, "cmp%d" % f)
        else:
            N = len(w["type_idx"])
            rms_err = np.sqrt(((one["force"] - ref["force"]) ** 2).mean())
            assert rms_err <= 5e-3 and rms_err <= 3e-2 * np.sqrt((ref["force"] ** 2).mean())
            assert abs(one["energy"] - ref["energy"]) / N <= 2e-2 * np.abs(ref["atom_energy"]).mean() + 1e-6


def test_compressed_tables_match_uncompressed_model():
    """The compressed form of model B on the 192-atom box: FP32 kernels vs the
    float64 oracle with the same tables, and vs the uncompressed float64
    model (the compression error of 256 intervals is far below the bars)."""
    from make_golden import hermite_compressed
    pc, vc = hermite_compressed(*MODELS["B"])
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    got = run_gpu(pc, vc, pos, box, typ)
    assert got["status"] == 0
    one = dict(energy=got["energy"][0], force=got["force"][0], virial=got["virial"][0],
               atom_energy=got["atom_energy"][0])
    check_close(one, om.energy_force(om.OracleModel(pc, vc, torch.float64), pos, box, typ), "cmp")
    ref = om.energy_force(om.OracleModel(*MODELS["B"], torch.float64), pos, box, typ)
    ref["energy"] = float(G["B_E"])
    check_close(one, ref, "cmp-vs-uncompressed")


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_empty_type_block_and_isolated_atoms(precision):
    """Edge cases of the evaluation in both forms: a box of oxygen only (the
    H type block of the two-type model is empty) against the FP64 oracle,
    and atoms with no neighbour within rcut (every environment empty):
    forces and virial exactly zero, each atom's energy the fitting net of a
    zero descriptor of its type."""
    from deepmd_jax_b200.systems import water_box
    p, v = MODELS["B"]
    m = om.OracleModel(p, v, torch.float64)
    w = water_box(8, 24.83, seed=21)
    oxy = w["type_idx"] == 0
    pos, typ = w["position"][oxy], w["type_idx"][oxy]
    got = run_gpu(p, v, pos, w["box"], typ, precision=precision)
    assert got["status"] == 0
    ref = om.energy_force(m, pos, w["box"], typ, nbrs=got["nbrs"][0], sel=[46, 92])
    if precision == "fp32":
        check_close(dict(energy=got["energy"][0], force=got["force"][0], virial=got["virial"][0],
                         atom_energy=got["atom_energy"][0]), ref, "O only")
    else:  # BF16 GEMMs: the tolerances of the mixed form
        rms = np.sqrt(((got["force"][0] - ref["force"]) ** 2).mean() / (ref["force"] ** 2).mean())
        assert rms <= 3e-2, rms
        assert abs(got["energy"][0] - ref["energy"]) <= 2e-2 * np.abs(ref["atom_energy"]).sum()
    pos2 = np.array([[1.0, 1.0, 1.0], [10.0, 10.0, 10.0], [20.0, 20.0, 1.0], [1.0, 20.0, 12.0]])
    typ2 = np.array([0, 1, 1, 0])
    got2 = run_gpu(p, v, pos2, w["box"], typ2, precision=precision)
    ref2 = om.energy_force(m, pos2, w["box"], typ2)
    assert got2["status"] == 0
    assert np.all(got2["force"] == 0.0) and np.all(got2["virial"] == 0.0)
    tol = 2e-6 if precision == "fp32" else 2e-2
    assert np.abs(got2["atom_energy"][0] - ref2["atom_energy"]).max() <= tol * np.abs(ref2["atom_energy"]).max()


def test_full_size_invariants_fp32_and_mixed():
    """The 98,304-atom benchmark box (32,768 waters, L = 99.3 A), benchmark
    model architecture: properties that hold at any size.  Two frames, the
    second a rigid translation by (0.37, -1.2, 2.9) A: energies within
    2e-6 x sum|E_atom| and forces within 2e-4 x max|F| of each other (FP32);
    the total force vanishes (<= 1e-5 x sum|F|); the energy is the sum of
    the atom energies; the virial is symmetric (<= 1e-4 x max|W|).  The
    mixed form against FP32 on the same lists: force RMS difference
    <= 5e-3 eV/A and <= 3e-2 x force RMS."""
    from deepmd_jax_b200.systems import init_dp_params, water_box
    from make_golden import randomize_model
    p, v = randomize_model(*init_dp_params(nnbrs=90.0, seed=0), seed=1)
    w = water_box(32, 99.3, seed=5)
    pos = np.stack([w["position"], w["position"] + np.array([0.37, -1.2, 2.9])])
    sel = (60, 120)
    r32 = run_gpu(p, v, pos, w["box"], w["type_idx"], sel=sel)
    assert r32["status"] == 0
    eabs = np.abs(r32["atom_energy"][0]).sum()
    assert abs(r32["energy"][0] - r32["energy"][1]) <= 2e-6 * eabs
    fmax = np.abs(r32["force"][0]).max()
    assert np.abs(r32["force"][0] - r32["force"][1]).max() <= 2e-4 * fmax
    for f in range(2):
        F = r32["force"][f].astype(np.float64)
        assert np.abs(F.sum(0)).max() <= 1e-5 * np.abs(F).sum()
        assert abs(r32["energy"][f] - r32["atom_energy"][f].sum()) <= 1e-6 * eabs
        W = r32["virial"][f]
        assert np.abs(W - W.T).max() <= 1e-4 * np.abs(W).max()
    rmx = run_gpu(p, v, pos, w["box"], w["type_idx"], sel=sel, precision="mixed")
    assert rmx["status"] == 0
    for f in range(2):
        d = rmx["force"][f] - r32["force"][f]
        rms_d = np.sqrt((d ** 2).mean())
        assert rms_d <= 5e-3 and rms_d <= 3e-2 * np.sqrt((r32["force"][f] ** 2).mean()), rms_d
