"""Chunk re-run after a hard overflow inside a chunk (deepmd_jax/md.py:905-916,
644-676): the chunk is discarded, the cause resolved, the chunk run again.

* Bit 2 (neighbour overflow): an engine whose capacity is the exact maximum
  neighbour count of the initial frame (buffer ratio 1.0) overflows at a
  drift-gated rebuild in the middle of a 40-step chunk.  It must reallocate
  and re-run that chunk, so its trajectory equals the one of an engine given
  the grown capacity from step 0; an engine that kept the truncated list for
  the rest of the chunk would miss pairs within rcut.
* Bit 1 (box shrank past the skin, NPT): a tiny skin makes the barostat's
  first box contraction trip the check; the skin grows by 0.4 A and the
  chunk re-runs, matching an engine started with the grown skin.

"Equals" is measured against the engine's own run-to-run spread: the force
scatter adds in float32 atomics, whose order varies from run to run, and the
random-init model (no short-range repulsion, atoms heat up and pass close to
one another) grows that last-bit noise by orders of magnitude at a close
approach (in this box one comes near step 55, where two clean runs part from
2e-6 A to 2e-4 A within three steps).  The runs stop at 40 steps, before it,
and a second engine with the grown setting gives the yardstick: the re-run
trajectory must lie within 1e-5 A over the first 10 steps and, after them,
within 10x the distance between the two clean runs or 1e-4 A, whichever is
larger.  The floor covers a last-bit difference that appears in one run and
not in the other (one float32 ulp of a coordinate near 24 A is 1.9e-6 A; one
such difference in a velocity grows by about 8e-6 A per step over the last
ten steps here).  A wrong re-run (a lost neighbour, a chunk that does not
restart from its saved state) moves atoms by a perturbation of a missing
pair's force: 1e-3 eV/A on a hydrogen for 30 steps of 0.5 fs displaces it by
about 1e-3 A, ten times the floor, and a chunk that does not restart differs
from the first frames on.
"""
import ctypes

import numpy as np
import pytest

from make_golden import golden_models

pytestmark = pytest.mark.gpu


def _water(n=8, L=24.83, seed=5):
    from deepmd_jax_b200.systems import water_box
    return water_box(n, L, seed=seed)


def _frame_diff(a, b):
    """Max |a - b| per frame of two trajectories' positions."""
    return np.abs(a["position"] - b["position"]).reshape(len(a["position"]), -1).max(1)


def _same_within_spread(name, got, ref, ref2):
    d = _frame_diff(got, ref)
    d0 = _frame_diff(ref, ref2)
    print("%s: re-run vs clean %.2e A (step 10: %.2e), clean vs clean %.2e A (step 10: %.2e)"
          % (name, d.max(), d[10], d0.max(), d0[10]))
    assert d[:11].max() < 1e-5
    assert d.max() <= max(10.0 * d0.max(), 1e-4)


def test_neighbour_overflow_mid_chunk_is_rerun_at_grown_capacity():
    from deepmd_jax_b200 import _lib
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _water()
    kw = dict(initial_velocity=w["velocity"], report_interval=200, verbose=False)
    tight = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                       neighbor_buffer_ratio=1.0, **kw)
    sel0 = list(tight._sel)
    traj_t = tight.run(40)
    sel1 = list(tight._sel)
    assert any(b > a for a, b in zip(sel0, sel1)), "the tight capacity never overflowed (%s)" % sel0
    assert tight.step == 40 and int(tight._report_struct().status) & 2 == 0

    def clean():
        sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"], **kw)
        arr = (ctypes.c_int * len(sel1))(*sel1)
        _lib.check(sim.lib.dpb_md_set_capacity(sim._h, arr, None), "dpb_md_set_capacity")
        sim._sel = sel1
        return sim.run(40)

    print("capacity %s -> %s" % (sel0, sel1))
    _same_within_spread("neighbour overflow", traj_t, clean(), clean())


def test_npt_box_shrink_past_skin_is_rerun_with_grown_skin():
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _water()
    kw = dict(initial_velocity=w["velocity"], temperature=300.0, pressure=1.0e4, tau_t=100.0, tau_p=100.0,
              report_interval=200, verbose=False)
    small = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.5, w["position"],
                       neighbor_skin=0.01, **kw)
    traj_s = small.run(40)
    assert small._neighbor_skin > 0.01 + 0.3, "the box never shrank past the 0.01 A skin"
    assert small.step == 40

    def clean():
        sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.5, w["position"],
                         neighbor_skin=small._neighbor_skin, **kw)
        return sim.run(40)

    g1, g2 = clean(), clean()
    print("skin 0.01 -> %.2f A; box difference %.2e A (clean vs clean %.2e A)"
          % (small._neighbor_skin, np.abs(traj_s["box"] - g1["box"]).max(), np.abs(g1["box"] - g2["box"]).max()))
    _same_within_spread("box shrink", traj_s, g1, g2)
