"""Model shapes beyond the tuned instantiations (golden_shapes.npz from the
reference source, make_golden_shapes.py) through the general FP32 kernels:
energy and forces against the golden vectors, with the FP32 form's bars
(energy <= 2e-6 sum|E_atom| + 1e-6 eV, forces <= 2e-4 of the largest
component), and the mixed form within its bars."""
import os

import numpy as np
import pytest
import torch

from gpu_helpers import run_gpu
from make_golden_shapes import shape_models

pytestmark = pytest.mark.gpu

GS = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_shapes.npz"))


def _case(key):
    mk = "F" if key == "L" else key
    p, v = shape_models()[mk]
    pre = "L_" if key == "L" else ""
    return p, v, GS[pre + "pos"], GS[pre + "box"], GS[pre + "type"]


@pytest.mark.parametrize("key", ["F", "G", "H", "I", "L"])
def test_general_shapes_fp32_match_reference(key):
    from oracle import model as om
    p, v, pos, box, typ = _case(key)
    out = run_gpu(p, v, pos, box, typ)
    assert out["status"] == 0
    ref_atoms = om.energy_force(om.OracleModel(p, v, torch.float64), pos, box, typ)["atom_energy"]
    E, F = float(GS[key + "_E"]), GS[key + "_F"]
    dE = abs(float(out["energy"][0]) - E)
    dF = np.abs(out["force"][0] - F).max() / np.abs(F).max()
    print("%s: |dE| %.2e eV, max |dF| / max |F| %.2e" % (key, dE, dF))
    assert dE <= 2e-6 * np.abs(ref_atoms).sum() + 1e-6
    assert dF <= 2e-4


@pytest.mark.parametrize("key", ["F", "G", "H", "I", "L"])
def test_general_shapes_mixed_form(key):
    """The mixed form on the same shapes: tensor-core fitting at the padded
    hidden width (208 for 200, 240 for 240-120-240, 64 for 64-64; zero padding
    is exact), FP32 embedding kernels (no tensor-core embedding for these
    shapes), within the mixed form's bars."""
    from oracle import model as om
    p, v, pos, box, typ = _case(key)
    out = run_gpu(p, v, pos, box, typ, precision="mixed")
    assert out["status"] == 0
    ref_atoms = om.energy_force(om.OracleModel(p, v, torch.float64), pos, box, typ)["atom_energy"]
    F = GS[key + "_F"]
    rms_err = np.sqrt(((out["force"][0] - F) ** 2).mean())
    rms_f = np.sqrt((F ** 2).mean())
    de = abs(float(out["energy"][0]) - float(GS[key + "_E"])) / len(ref_atoms)
    print("%s mixed: force rms err %.2e (rel %.2e), energy/atom err %.2e" % (key, rms_err, rms_err / rms_f, de))
    assert rms_err <= 5e-3 and rms_err <= 3e-2 * rms_f
    assert de <= 2e-2 * np.abs(ref_atoms).mean()
