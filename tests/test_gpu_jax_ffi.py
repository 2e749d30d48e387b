"""The jax.ffi custom calls (csrc/jax_ffi/dpb_jax_ffi.cc) against the ctypes
path on a 1,536-atom water box: the neighbour list bit for bit, energy /
force / virial to FP32 summation-order noise.  Needs jax with its FFI
headers; where jax is absent (this image) the test skips."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_jax_ffi_eval_matches_ctypes_path():
    jax = pytest.importorskip("jax")
    pytest.importorskip("jax.ffi")
    import jax.numpy as jnp
    from make_golden import golden_models
    from gpu_helpers import run_gpu
    from deepmd_jax_b200 import jax_ffi
    from deepmd_jax_b200.engine import DeviceModel, sort_by_type
    from deepmd_jax_b200.systems import water_box
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "deepmd-jax_b200", "csrc", "jax_ffi")])
    jax.config.update("jax_enable_x64", True)
    p, v = golden_models()["B"]
    w = water_box(8, 24.83, seed=3)
    dm = DeviceModel(p, v)
    perm, cnt = sort_by_type(w["type_idx"], 2)
    sel = [46, 92]
    ref = run_gpu(p, v, w["position"], w["box"], w["type_idx"], sel=sel, device_model=dm)
    pos = jnp.asarray(w["position"][None], jnp.float32)
    pm = jnp.asarray(perm, jnp.int32)
    nb, _, st = jax_ffi.nlist_build(pos, pm, w["box"], 6.3, cnt, sel, 64 << 20)
    assert int(st[0]) == 0
    assert np.array_equal(np.asarray(nb), ref["nbrs"])
    ws = dm.eval_workspace(len(perm), 1).numel()
    E, F, W, st = jax_ffi.energy_and_force(pos, pm, jnp.asarray(w["box"][None], jnp.float32), nb, dm.handle.value,
                                           cnt, sel, ws)
    assert int(st[0]) == 0
    assert abs(float(E[0]) - float(ref["energy"][0])) < 1e-6 * max(1.0, abs(float(ref["energy"][0])))
    assert np.abs(np.asarray(F) - ref["force"]).max() <= 1e-5 * np.abs(ref["force"]).max()
    assert np.abs(np.asarray(W).reshape(1, 3, 3) - ref["virial"]).max() <= 1e-5 * np.abs(ref["virial"]).max()
