"""NVE energy conservation of the mixed form against the plain FP32 form on
the 192-atom water box with the benchmark model (random init), over the first
100 steps (dt 0.5 fs), total energy sampled at every step.

The random-init model has no short-range repulsion: atoms pass through one
another, and each such pass (s(r) = 1/r grows without bound) kicks the total
energy by far more than any rounding - the float64 oracle integrator shows the
same jumps from step ~120 on.  The first 100 steps are free of such passes, so
the total energy there measures the integrator and the force/energy
consistency of each form.

Target: "NVE drift no worse than the plain form".  The drift is the
least-squares slope of E_total / N in eV/atom/ps; the mixed slope must not
exceed the FP32 slope by more than three standard errors of the mixed fit
(its energy carries 16-bit GEMM rounding noise, so its slope estimate is
noisier) plus 1e-6 eV/atom/ps.  Also both stay within 1e-5 eV/atom of E(0).
"""
import numpy as np
import pytest

from make_golden import golden_models

pytestmark = pytest.mark.gpu


def _trace(precision, nsteps=100):
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["A"]
    w = water_box(4, 12.42, seed=0)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], report_interval=1, precision=precision, verbose=False)
    sim.run(nsteps, trajectory=False)
    t_ps = np.array([row[0] for row in sim.log]) * 0.5e-3
    e = np.array([row[4] for row in sim.log]) / 192
    A = np.stack([t_ps, np.ones_like(t_ps)], 1)
    coef = np.linalg.lstsq(A, e, rcond=None)[0]
    resid = e - A @ coef
    se = np.sqrt((resid ** 2).sum() / (len(e) - 2) / ((t_ps - t_ps.mean()) ** 2).sum())
    return np.abs(e - e[0]).max(), coef[0], se, len(e)


def test_nve_drift_mixed_no_worse_than_fp32():
    d32, s32, se32, n = _trace("fp32")
    dmx, smx, semx, _ = _trace("mixed")
    print("\nNVE 100 steps, %d samples: max |E(t)-E(0)|/N fp32 %.3e mixed %.3e eV/atom; drift fp32 %.3e "
          "(se %.1e) mixed %.3e (se %.1e) eV/atom/ps" % (n, d32, dmx, s32, se32, smx, semx))
    assert n == 101
    assert d32 <= 1e-5 and dmx <= 1e-5
    assert abs(smx) <= abs(s32) + 3.0 * semx + 1e-6
