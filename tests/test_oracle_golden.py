"""The oracle against golden vectors produced by the reference's own model
source (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest
import torch

from make_golden import golden_models
from oracle import model as om

G = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "golden_model.npz"))
MODELS = golden_models()

CASES = [("A", "A", "A", None), ("B", "A", "B", None), ("C", "A", "C", None),
         ("D", "D", "B", "D_nbrs"), ("E", "E", "B", None)]


@pytest.mark.parametrize("key,sysk,mk,nb", CASES)
def test_oracle_matches_reference_source(key, sysk, mk, nb):
    p, v = MODELS[mk]
    m = om.OracleModel(p, v, torch.float64)
    r = om.energy_force(m, G[sysk + "_pos"], G[sysk + "_box"], G[sysk + "_type"],
                        nbrs=(G[nb] if nb else None), sel=[46, 92])
    assert abs(r["energy"] - float(G[key + "_E"])) <= 1e-12 * max(1.0, abs(float(G[key + "_E"])))
    assert np.abs(r["force"] - G[key + "_F"]).max() <= 1e-12


def test_oracle_force_is_gradient():
    """Central finite differences of the oracle energy (h = 1e-4 A)."""
    p, v = MODELS["B"]
    m = om.OracleModel(p, v, torch.float64)
    pos, box, typ = G["A_pos"], G["A_box"], G["A_type"]
    F = om.energy_force(m, pos, box, typ)["force"]
    rng = np.random.default_rng(0)
    for _ in range(6):
        a, c = rng.integers(len(pos)), rng.integers(3)
        h = 1e-4
        pp = pos.copy(); pp[a, c] += h
        pm = pos.copy(); pm[a, c] -= h
        fd = -(om.energy_only(m, pp, box, typ)[0] - om.energy_only(m, pm, box, typ)[0]) / (2 * h)
        assert abs(fd - F[a, c]) < 1e-7


def test_oracle_virial_trace_is_strain_derivative():
    p, v = MODELS["B"]
    m = om.OracleModel(p, v, torch.float64)
    pos, box, typ = G["E_pos"], G["E_box"], G["E_type"]
    W = om.energy_force(m, pos, box, typ)["virial"]
    eps = 1e-6
    ep = om.energy_only(m, pos * (1 + eps), box * (1 + eps), typ)[0]
    em = om.energy_only(m, pos * (1 - eps), box * (1 - eps), typ)[0]
    assert abs((ep - em) / (2 * eps) + np.trace(W)) < 1e-6
    assert np.abs(W - W.T).max() < 1e-10      # rotation invariance -> symmetric


def test_normal_modes_match_reference_source():
    """Ring-polymer normal modes of the reference's pimd.normal_mode_transform
    (deepmd_jax/pimd.py:22-44, P = 8 at 300 K, golden fixture) against the
    oracle's and the product host's: frequencies to 1e-12 relative; C
    orthogonal; and, since eigenvectors of a degenerate pair are defined
    only up to a rotation, the same projector onto each frequency's modes."""
    from deepmd_jax_b200.md import normal_mode_transform as host_nm
    from oracle import integrators as oi
    P, kT = 8, 300.0 * 8.617333e-5
    fg, Cg = G["pimd_freqs"], G["pimd_C"]
    for freqs, C in (oi.normal_mode_transform(P, kT), host_nm(P, kT)):
        assert np.allclose(freqs, fg, rtol=1e-12, atol=1e-15)
        assert np.allclose(C.T @ C, np.eye(P), atol=1e-12)
        for f in np.unique(np.round(fg, 12)):
            sel = np.isclose(fg, f, rtol=1e-9, atol=1e-15)
            assert np.allclose(C[:, sel] @ C[:, sel].T, Cg[:, sel] @ Cg[:, sel].T, atol=1e-12)


GS = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "golden_shapes.npz"))


@pytest.mark.parametrize("key", ["F", "G", "H", "I", "L"])
def test_oracle_matches_reference_source_other_shapes(key):
    """Embedding / fitting shapes beyond the benchmark's (make_golden_shapes.py):
    (24,48,96)/(200,200,200)/axis 12, (16,32,64)/(240,120,240), a four-layer
    net with a narrowing layer, a compressed width-96 table, and F through a
    neighbour list."""
    from make_golden_shapes import shape_models
    mk = "F" if key == "L" else key
    p, v = shape_models()[mk]
    m = om.OracleModel(p, v, torch.float64)
    pre = "L_" if key == "L" else ""
    r = om.energy_force(m, GS[pre + "pos"], GS[pre + "box"], GS[pre + "type"],
                        nbrs=(GS["L_nbrs"] if key == "L" else None), sel=[46, 92])
    assert abs(r["energy"] - float(GS[key + "_E"])) <= 1e-12 * max(1.0, abs(float(GS[key + "_E"])))
    assert np.abs(r["force"] - GS[key + "_F"]).max() <= 1e-12
