"""Chunk re-run after a hard overflow inside a chunk (deepmd_jax/md.py:905-916,
644-676): the chunk is discarded, the cause resolved, the chunk run again.

* Bit 2 (neighbour overflow): an engine whose capacity is the exact maximum
  neighbour count of the initial frame (buffer ratio 1.0) overflows at a
  drift-gated rebuild in the middle of a 60-step chunk.  It must reallocate
  and re-run that chunk, so its trajectory equals (to FP32 summation noise)
  the one of an engine given the grown capacity from step 0; an engine that
  kept the truncated list for the rest of the chunk would miss pairs within
  rcut and drift away by orders of magnitude more.
* Bit 1 (box shrank past the skin, NPT): a tiny skin makes the barostat's
  first box contraction trip the check; the skin grows by 0.4 A and the
  chunk re-runs, matching an engine started with the grown skin.
"""
import ctypes

import numpy as np
import pytest

from make_golden import golden_models

pytestmark = pytest.mark.gpu


def _water(n=8, L=24.83, seed=5):
    from deepmd_jax_b200.systems import water_box
    return water_box(n, L, seed=seed)


def test_neighbour_overflow_mid_chunk_is_rerun_at_grown_capacity():
    from deepmd_jax_b200 import _lib
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _water()
    kw = dict(initial_velocity=w["velocity"], report_interval=200, verbose=False)
    tight = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                       neighbor_buffer_ratio=1.0, **kw)
    sel0 = list(tight._sel)
    traj_t = tight.run(60)
    sel1 = list(tight._sel)
    assert any(b > a for a, b in zip(sel0, sel1)), "the tight capacity never overflowed (%s)" % sel0
    assert tight.step == 60 and int(tight._report_struct().status) & 2 == 0
    roomy = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"], **kw)
    arr = (ctypes.c_int * len(sel1))(*sel1)
    _lib.check(roomy.lib.dpb_md_set_capacity(roomy._h, arr, None), "dpb_md_set_capacity")
    roomy._sel = sel1
    traj_r = roomy.run(60)
    err = np.abs(traj_t["position"] - traj_r["position"]).max()
    print("capacity %s -> %s; trajectory difference %.2e A" % (sel0, sel1, err))
    assert err < 1e-5


def test_npt_box_shrink_past_skin_is_rerun_with_grown_skin():
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _water()
    kw = dict(initial_velocity=w["velocity"], temperature=300.0, pressure=1.0e4, tau_t=100.0, tau_p=100.0,
              report_interval=200, verbose=False)
    small = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.5, w["position"],
                       neighbor_skin=0.01, **kw)
    traj_s = small.run(60)
    assert small._neighbor_skin > 0.01 + 0.3, "the box never shrank past the 0.01 A skin"
    assert small.step == 60
    grown = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.5, w["position"],
                       neighbor_skin=small._neighbor_skin, **kw)
    traj_g = grown.run(60)
    err = np.abs(traj_s["position"] - traj_g["position"]).max()
    berr = np.abs(traj_s["box"] - traj_g["box"]).max()
    print("skin 0.01 -> %.2f A; trajectory difference %.2e A, box %.2e A" % (small._neighbor_skin, err, berr))
    assert err < 1e-5 and berr < 1e-6
