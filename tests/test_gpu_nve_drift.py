"""NVE energy conservation of the mixed form against the plain FP32 form on
the 192-atom water box with the benchmark model (random init), over the first
100 steps (dt 0.5 fs), sampled at every step.

The random-init model has no short-range repulsion: atoms pass through one
another, and each such pass (s(r) = 1/r grows without bound) kicks the total
energy by far more than any rounding - the float64 oracle integrator shows the
same jumps from step ~120 on.  The first 100 steps are free of such passes, so
the total energy there measures the integrator and the force/energy
consistency of each form.

Two energies are followed along each form's trajectory:

* the form's own total energy (its potential energy + kinetic energy), the
  quantity its integrator conserves.  The drift is the least-squares slope
  of E_total / N in eV/atom/ps, and "no worse than the plain form" means: the
  mixed slope exceeds the FP32 slope by at most three standard errors of the
  mixed fit plus 1e-6 eV/atom/ps;
* the float64 Hamiltonian: the float64 oracle's potential energy of every
  frame + the kinetic energy of the frame's velocities.  The mixed form's
  FP16 weights make it a slightly different potential (forces off by ~1e-4
  of their size on this model), and the difference changes as the random
  model's potential energy turns into heat, so this slope is held to a
  bound, 1e-5 eV/atom/ps, not to the FP32 figure.

Both forms also stay within 1e-5 eV/atom of E(0) in their own energy.
"""
import numpy as np
import pytest
import torch

from make_golden import golden_models
from oracle import integrators as oi
from oracle import model as om

pytestmark = pytest.mark.gpu

MU = 1.036427e2


def _slope(t_ps, e):
    A = np.stack([t_ps, np.ones_like(t_ps)], 1)
    coef = np.linalg.lstsq(A, e, rcond=None)[0]
    resid = e - A @ coef
    se = np.sqrt((resid ** 2).sum() / (len(e) - 2) / ((t_ps - t_ps.mean()) ** 2).sum())
    return coef[0], se


def _trace(precision, m64, nsteps=100):
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["A"]
    w = water_box(4, 12.42, seed=0)
    N = len(w["type_idx"])
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], report_interval=1, precision=precision, verbose=False)
    traj = sim.run(nsteps)
    t_ps = np.array([row[0] for row in sim.log]) * 0.5e-3
    e_rep = np.array([row[4] for row in sim.log]) / N
    mass = (w["mass"] * MU)[:, None]
    e64 = []
    for r, vel in zip(traj["position"], traj["velocity"]):
        pe = om.energy_force(m64, r, w["box"], w["type_idx"], virial=False)["energy"]
        e64.append(float(pe) + oi.kinetic_energy(vel * mass, mass))
    e64 = np.array(e64) / N
    t64 = np.arange(len(e64)) * 0.5e-3
    s_rep, se_rep = _slope(t_ps, e_rep)
    s64, se64 = _slope(t64, e64)
    return dict(n=len(e_rep), dev_rep=np.abs(e_rep - e_rep[0]).max(), s_rep=s_rep, se_rep=se_rep,
                n64=len(e64), dev64=np.abs(e64 - e64[0]).max(), s64=s64, se64=se64)


def test_nve_drift_mixed_no_worse_than_fp32():
    p, v = golden_models()["A"]
    m64 = om.OracleModel(p, v, torch.float64, device="cuda")
    a = _trace("fp32", m64)
    b = _trace("mixed", m64)
    for name, r in (("fp32", a), ("mixed", b)):
        print("\nNVE 100 steps %s: reported max |E-E0|/N %.3e, slope %.3e (se %.1e); float64 Hamiltonian max "
              "|H-H0|/N %.3e, slope %.3e (se %.1e) eV/atom/ps"
              % (name, r["dev_rep"], r["s_rep"], r["se_rep"], r["dev64"], r["s64"], r["se64"]))
    assert a["n"] == 101 and b["n"] == 101 and a["n64"] == 101 and b["n64"] == 101
    assert a["dev_rep"] <= 1e-5 and b["dev_rep"] <= 1e-5
    assert abs(b["s_rep"]) <= abs(a["s_rep"]) + 3.0 * b["se_rep"] + 1e-6
    assert abs(b["s64"]) <= 1e-5
