"""Mixed form (BF16 tcgen05 GEMMs, FP32 accumulation) against the FP32 path
and the float64 oracle.

Tolerances for the mixed form (stated, checked): descriptor T and G within
2e-2 of their max magnitude of the FP32 path; energy per atom within 2e-2 of
the mean |E_atom|; forces: RMS error / RMS force <= 3e-2, and absolute RMS
error <= 5e-3 eV/A (the target of the mixed form).
"""
import ctypes
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


def _descriptors(precision, p, v, w):
    from deepmd_jax_b200 import _lib
    from deepmd_jax_b200.engine import DeviceModel, NeighborBuilder, sort_by_type, _ptr, _stream
    dm = DeviceModel(p, v)
    lib = dm.lib
    lib.dpb_eval_descriptors.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 2 + \
        [ctypes.c_int] * 2 + [ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.POINTER(ctypes.c_int)] + [ctypes.c_void_p] * 4 + \
        [ctypes.c_size_t, ctypes.c_void_p]
    perm, cnt = sort_by_type(w["type_idx"], 2)
    N = len(perm)
    pos = torch.tensor(np.ascontiguousarray(w["position"][None]), dtype=torch.float32, device="cuda")
    pm = torch.tensor(perm, dtype=torch.int32, device="cuda")
    box = torch.tensor(np.ascontiguousarray(w["box"][None]), dtype=torch.float32, device="cuda")
    nbrs, _ = NeighborBuilder(N, 1, cnt, [46, 92], w["box"], 6.3).build(pos, perm=pm)
    W, A = p["embed_widths"][-1], p["axis"]
    T = torch.zeros((N, 10, W), dtype=torch.float32, device="cuda")
    Gd = torch.zeros((N, A * W), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws = dm.eval_workspace(N, 1)
    rc = lib.dpb_eval_descriptors(dm.handle, {"fp32": 0, "mixed": 1}[precision], _ptr(pos), _ptr(pm), N, 1,
                                  _lib.int_array(cnt), _ptr(box), _ptr(nbrs), _lib.int_array([46, 92]), _ptr(T),
                                  _ptr(Gd), _ptr(err), _ptr(ws), ws.numel(), _stream())
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    return T.cpu().numpy(), Gd.cpu().numpy()


@pytest.mark.parametrize("mk", ["A", "B"])
def test_mixed_descriptors_match_fp32(mk):
    from deepmd_jax_b200.systems import water_box
    p, v = MODELS[mk]
    w = water_box(8, 24.83, seed=7)
    T32, G32 = _descriptors("fp32", p, v, w)
    Tm, Gm = _descriptors("mixed", p, v, w)
    assert np.abs(Tm - T32).max() <= 2e-2 * np.abs(T32).max()
    assert np.abs(Gm - G32).max() <= 2e-2 * np.abs(G32).max()


@pytest.mark.parametrize("key,sysk,mk", [("B", "A", "B"), ("D", "D", "B"), ("A", "A", "A"), ("H", "A", "H")])
def test_mixed_eval_vs_fp64(key, sysk, mk):
    """H: model B with compressed (C2 piecewise quintic) embedding tables."""
    if mk == "H":
        from make_golden import hermite_compressed
        p, v = hermite_compressed(*MODELS["B"])
    else:
        p, v = MODELS[mk]
    pos, box, typ = G[sysk + "_pos"], G[sysk + "_box"], G[sysk + "_type"]
    got = run_gpu(p, v, pos, box, typ, precision="mixed")
    assert got["status"] == 0
    ref = om.energy_force(om.OracleModel(p, v, torch.float64), pos, box, typ)
    N = len(typ)
    dF = got["force"][0] - ref["force"]
    rms_err = np.sqrt((dF ** 2).mean())
    rms_f = np.sqrt((ref["force"] ** 2).mean())
    e_err = abs(got["energy"][0] - ref["energy"]) / N
    print("mixed %s: force rms err %.3e (rel %.3e), energy/atom err %.3e" % (key, rms_err, rms_err / rms_f, e_err))
    assert rms_err <= 5e-3
    assert rms_err <= 3e-2 * rms_f
    assert e_err <= 2e-2 * np.abs(ref["atom_energy"]).mean() + 1e-6


def test_mixed_default_train_widths():
    """The reference train() default architecture (embed 32-32-64, fit 128^3,
    axis 12; deepmd_jax/train.py:24-27) in the mixed form, against FP64."""
    from deepmd_jax_b200.systems import water_box, init_dp_params
    from make_golden import randomize_model
    w = water_box(8, 24.83, seed=5)
    p, v = randomize_model(*init_dp_params(embed_widths=(32, 32, 64), fit_widths=(128, 128, 128), axis=12,
                                           nnbrs=90.0, seed=3), seed=4)
    got = run_gpu(p, v, w["position"], w["box"], w["type_idx"], precision="mixed")
    assert got["status"] == 0
    ref = om.energy_force(om.OracleModel(p, v, torch.float64), w["position"], w["box"], w["type_idx"],
                          nbrs=got["nbrs"][0], sel=[46, 92])
    N = len(w["type_idx"])
    rms_err = np.sqrt(((got["force"][0] - ref["force"]) ** 2).mean())
    rms_f = np.sqrt((ref["force"] ** 2).mean())
    print("mixed default widths: force rms err %.3e (rel %.3e)" % (rms_err, rms_err / rms_f))
    assert rms_err <= 5e-3 and rms_err <= 3e-2 * rms_f
    assert abs(got["energy"][0] - ref["energy"]) / N <= 2e-2 * np.abs(ref["atom_energy"]).mean() + 1e-6
