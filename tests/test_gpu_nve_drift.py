"""NVE energy conservation of the FP32 and mixed forms on the 192-atom water
box with the benchmark model (random init), over the first 100 steps
(dt 0.5 fs).

The random-init model has no short-range repulsion: atoms pass through one
another, and each such pass (s(r) = 1/r grows without bound) kicks the total
energy by far more than any rounding - the float64 oracle integrator shows the
same jumps from step ~120 on.  The first 100 steps are free of such passes, so
the total energy there measures the integrator and the force/energy
consistency of each form.

Bars: max |E(t) - E(0)| / N <= 1e-5 eV/atom and |drift| (least-squares slope)
<= 1e-4 eV/atom/ps for both forms.  The mixed form's energy fluctuates more
than the FP32 form's (its per-atom energies carry BF16 rounding, ~1e-6 eV);
the test prints both.
"""
import numpy as np
import pytest

from make_golden import golden_models

pytestmark = pytest.mark.gpu


def _trace(precision):
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["A"]
    w = water_box(4, 12.42, seed=0)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], report_interval=10, precision=precision, verbose=False)
    sim.run(100, trajectory=False)
    t_ps = np.array([row[0] for row in sim.log]) * 0.5e-3
    e = np.array([row[4] for row in sim.log]) / 192
    return np.abs(e - e[0]).max(), np.polyfit(t_ps, e, 1)[0], len(e)


def test_nve_energy_conservation_fp32_and_mixed():
    d32, s32, n = _trace("fp32")
    dmx, smx, _ = _trace("mixed")
    print("\nNVE 100 steps: max |E(t)-E(0)|/N fp32 %.3e mixed %.3e eV/atom; drift fp32 %.3e mixed %.3e "
          "eV/atom/ps (%d samples)" % (d32, dmx, s32, smx, n))
    assert n == 11
    assert d32 <= 1e-5 and dmx <= 1e-5
    assert abs(s32) <= 1e-4 and abs(smx) <= 1e-4
