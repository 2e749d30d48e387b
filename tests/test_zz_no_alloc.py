"""The allocation-free evaluation entry point, dpb_eval_noalloc.

It exists for callers that cannot allocate device memory (a host code with a
fixed memory pool, a plugin in a process that forbids foreign cudaMalloc):
its scratch is a fixed 64 MiB array inside the library on each device.  These
tests call it through the C ABI and check, on two calls in a row with
different inputs, that it returns what dpb_eval (caller workspace) returns,
in both precision forms (the FP32 and the mixed form carve different layouts
from the same array), within the tolerances of the other GPU tests of each
form; and that a system whose
workspace exceeds the array is rejected before any device work.  The file
sorts last so a stop-at-first-failure run has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from deepmd_jax_b200.systems import water_box
from make_golden import golden_models

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _noalloc(dm, pos, box, nbrs, cnt, sel, perm, prec="fp32"):
    from deepmd_jax_b200 import _lib
    F, N = pos.shape[:2]
    out = dict(energy=torch.empty(F, dtype=torch.float64, device="cuda"),
               force=torch.empty((F, N, 3), dtype=torch.float32, device="cuda"),
               virial=torch.empty((F, 9), dtype=torch.float64, device="cuda"),
               atom_energy=torch.empty((F, N), dtype=torch.float32, device="cuda"),
               status=torch.zeros(1, dtype=torch.int32, device="cuda"))
    code = _lib.PREC_FP32 if prec == "fp32" else _lib.PREC_MIXED
    rc = dm.lib.dpb_eval_noalloc(dm.handle, code, _ptr(pos), _ptr(perm), N, F, _lib.int_array(cnt),
                                 _ptr(box), _ptr(nbrs), _lib.int_array(sel), _ptr(out["energy"]),
                                 _ptr(out["atom_energy"]), _ptr(out["force"]), _ptr(out["virial"]),
                                 _ptr(out["status"]), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, out


@pytest.mark.parametrize("prec", ["fp32", "mixed"])
def test_noalloc_matches_workspace_entry_on_two_calls(prec):
    from deepmd_jax_b200.engine import DeviceModel, NeighborBuilder, sort_by_type
    p, v = golden_models()["B"]
    dm = DeviceModel(p, v)
    sel = [46, 92]
    for seed in (21, 22):
        w = water_box(8, 24.83, seed=seed)
        perm, cnt = sort_by_type(w["type_idx"], 2)
        pos = torch.tensor(np.ascontiguousarray(w["position"][None]), dtype=torch.float32, device="cuda")
        pm = torch.tensor(perm, dtype=torch.int32, device="cuda")
        box = torch.tensor(np.ascontiguousarray(w["box"][None]), dtype=torch.float32, device="cuda")
        nbrs, _ = NeighborBuilder(len(perm), 1, cnt, sel, w["box"], 6.3).build(pos, perm=pm)
        ref = dm.evaluate(pos, box, nbrs, cnt, sel, perm=pm, atom_energy=True, precision=prec)
        rc, got = _noalloc(dm, pos, box, nbrs, cnt, sel, pm, prec)
        torch.cuda.synchronize()
        assert rc == 0
        assert int(got["status"].item()) == 0
        if prec == "mixed":  # the mixed form's bars (force RMS, energy per atom)
            f_ref, f_got = ref["force"].cpu().numpy(), got["force"].cpu().numpy()
            rms_err = np.sqrt(((f_got - f_ref) ** 2).mean())
            assert rms_err <= 5e-3 and rms_err <= 3e-2 * np.sqrt((f_ref ** 2).mean())
            a_ref = ref["atom_energy"].cpu().numpy()
            de = abs(float(got["energy"][0]) - float(ref["energy"][0])) / a_ref.size
            assert de <= 2e-2 * np.abs(a_ref).mean()
            continue
        e_ref, e_got = float(ref["energy"][0]), float(got["energy"][0])
        eabs = float(ref["atom_energy"].abs().sum())
        assert abs(e_got - e_ref) <= 2e-6 * eabs + 1e-6
        f_ref, f_got = ref["force"].cpu().numpy(), got["force"].cpu().numpy()
        assert np.abs(f_got - f_ref).max() <= 2e-4 * np.abs(f_ref).max()
        w_ref, w_got = ref["virial"].cpu().numpy(), got["virial"].cpu().numpy()
        assert np.abs(w_got - w_ref).max() <= 2e-4 * np.abs(w_ref).max() + 1e-9
        a_ref, a_got = ref["atom_energy"].cpu().numpy(), got["atom_energy"].cpu().numpy()
        assert np.abs(a_got - a_ref).max() <= 2e-6 * np.abs(a_ref).max() + 1e-6


def test_noalloc_rejects_systems_beyond_its_scratch():
    from deepmd_jax_b200 import _lib
    from deepmd_jax_b200.engine import DeviceModel
    p, v = golden_models()["B"]
    dm = DeviceModel(p, v)
    N = 12288                        # ~20 KB of workspace per atom, far beyond 64 MiB
    cnt, sel = [N // 3, 2 * N // 3], [46, 92]
    pos = torch.zeros((1, N, 3), dtype=torch.float32, device="cuda")
    box = torch.full((1, 3), 49.66, dtype=torch.float32, device="cuda")
    nbrs = torch.full((1, N, sum(sel)), N, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(dm, pos, box, nbrs, cnt, sel, None)
    assert rc == 261  # DPB_ERR_SCRATCH_LIMIT
    assert _lib.ERRORS[rc] == "DPB_ERR_SCRATCH_LIMIT"
