"""MD in neighbour-list mode (boxes wider than 2 (rcut + skin)), the mode the
benchmark runs, against the float64 oracle integrators.

* 1,536-atom water NVE, 60 steps, and 12,288-atom water NVT Nose-Hoover (the
  12,288-atom workload: benchmark model, 300 K, dt 0.5 fs), 100 steps, each
  checked three ways:
  - the device's rebuild steps vs the reference's soft-update rule
    (deepmd_jax/md.py:697-739) replayed on the device trajectory: rebuild at
    step t when the max minimum-image drift of the canonical positions after
    step t - 1 since the last rebuild exceeds ((rcut + skin) - rcut) / 2 -
    1e-6 min(box), all in float32 as the reference computes it;
  - every step against one float64 oracle step taken from the device's own
    state before it (positions, velocities and, for NVT, the chain
    variables): this holds each step, rebuild steps included, to float32
    rounding, where a whole-trajectory comparison cannot - the random-init
    models have no short-range repulsion, atoms heat up and pass close to one
    another, and the float32/float64 difference of the first steps grows by
    orders of magnitude within tens of steps (the float64 and float32 oracles
    part the same way);
  - the first 10 steps against the float64 oracle trajectory from the same
    initial state.
  Bars: per step 1e-5 A in position (a few float32 ulp of coordinates up to
  50 A) and 5e-5 of the largest speed in velocity (float32 forces of atoms in
  close approach); 1e-4 A after 10 steps; chain variables to 1e-4 of their
  largest magnitude.  A thermostat or integrator error of the size of one
  term (dt / tau_t = 5e-3 of the momenta per step) lands orders of magnitude
  outside.
* 32 beads x 1,536-atom water PILE-L (the path-integral workload: dt 0.25 fs,
  300 K), two steps vs the FP64 oracle with the same Philox noise.

The FP64 checker for the two large systems runs the oracle's torch code on
the GPU (float64) with a periodic k-d tree neighbour list (scipy), so the
tests finish in seconds; its energy does not depend on which list it uses as
long as every pair within rcut is present.
"""
import numpy as np
import pytest
import torch
from scipy.spatial import cKDTree

from make_golden import golden_models
from oracle import integrators as oi
from oracle import model as om
from oracle import nlist as onl
from oracle import philox

pytestmark = pytest.mark.gpu

MU = 1.036427e2
KB = 8.617333e-5
f32 = np.float32


def kd_nlist(pos, box, type_idx, rc, sel):
    """Typed block list (type-local ascending indices, pad N) of every pair
    closer than rc, from a periodic k-d tree on the type-sorted atoms."""
    perm, cnt = om.sort_by_type(type_idx, 2)
    cs = np.mod(np.asarray(pos, np.float64)[perm], box)
    cs = np.where(cs >= box, 0.0, cs)
    pairs = cKDTree(cs, boxsize=box).query_pairs(rc, output_type="ndarray")
    N = len(cs)
    i = np.concatenate([pairs[:, 0], pairs[:, 1]])
    j = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    offs, col = [0, cnt[0], N], [0, sel[0], sel[0] + sel[1]]
    out = np.full((N, sum(sel)), N, np.int32)
    for t in range(2):
        m = (j >= offs[t]) & (j < offs[t + 1])
        it, jt = i[m], j[m] - offs[t]
        rank = np.arange(len(it)) - np.searchsorted(it, np.arange(N))[it]
        assert rank.max(initial=-1) < sel[t], "oracle list capacity"
        out[it, col[t] + rank] = jt
    return out


def oracle_force_fn(m, box, type_idx, rc=6.5, sel=(80, 160)):
    def f(r):
        nb = kd_nlist(r, box, type_idx, rc, sel)
        out = om.energy_force(m, r, box, type_idx, nbrs=nb, sel=list(sel), virial=False)
        return out["force"], out["energy"]
    return f


def rebuild_steps_by_rule(traj_pos, box, type_idx, rcut, skin):
    """Steps t >= 1 at which the reference's soft update rebuilds, replayed in
    float32 on the device's trajectory (traj_pos[t] = positions after step t)."""
    box32 = np.asarray(box, f32)
    thr = f32(f32(f32(f32(rcut) + f32(skin)) - f32(rcut)) / f32(2)) - f32(box32.min()) * f32(1e-6)
    perm = np.argsort(np.asarray(type_idx), kind="stable")
    ref = onl.canonicalize(traj_pos[0], box32, type_idx)
    steps, margins = [], []
    for t in range(1, len(traj_pos)):
        now = onl.jnp_mod(np.asarray(traj_pos[t - 1], f32), box32)[perm]
        d = onl.max_drift(now, ref, box32)
        margins.append(abs(d - float(thr)))
        if f32(d) > thr:
            steps.append(t)
            ref = onl.canonicalize(traj_pos[t - 1], box32, type_idx)
    return steps, min(margins)


def run_stepwise(sim, nsteps):
    """One step per run() call: positions / velocities / Nose-Hoover chain
    (xi, p) after every step and the steps at which the engine rebuilt its
    list."""
    r0 = sim._report_struct()
    pos, vel, rebuilt = [sim.getPosition()], [sim.getVelocity()], []
    chain = [(np.array(r0.chain_xi[:3]), np.array(r0.chain_p[:3]))]
    n0 = int(r0.rebuilds)
    for t in range(1, nsteps + 1):
        tr = sim.run(1)
        pos.append(tr["position"][-1])
        vel.append(tr["velocity"][-1])
        r = sim._report_struct()
        chain.append((np.array(r.chain_xi[:3]), np.array(r.chain_p[:3])))
        n = int(r.rebuilds)
        if n > n0:
            rebuilt.append(t)
        n0 = n
    return np.array(pos), np.array(vel), rebuilt, chain


def shadow_errors(pos, vel, mass, box, fn, step):
    """Max position / velocity error of every device step against one float64
    oracle step from the device state before it.  fn(r) -> forces; step(r,
    p, F, F_next, t) -> (r, p) is one oracle step whose end-of-step force is
    F_next (the force at the device's next positions: the oracle's own next
    positions differ from them by float32 rounding, far below what the force
    can resolve)."""
    Fs = [fn(r) for r in pos]
    ep, ev = [], []
    for t in range(len(pos) - 1):
        r1, p1 = step(pos[t], vel[t] * mass, Fs[t], Fs[t + 1], t)
        ep.append(np.abs(oi.min_image_unwrap(r1, pos[t + 1], box) - r1).max())
        ev.append(np.abs(vel[t + 1] - p1 / mass).max())
    return np.array(ep), np.array(ev)


def _check_rebuilds(pos, w, sim, rebuilt, min_rebuilds):
    want, margin = rebuild_steps_by_rule(pos, w["box"], w["type_idx"], float(sim._params["rcut"]),
                                         sim._neighbor_skin)
    print("rebuild steps: device %s, rule %s (closest drift to the threshold %.2e A)" % (rebuilt, want, margin))
    assert len(want) >= min_rebuilds
    if margin > 1e-6:  # no decision within float32 reach of the threshold
        assert rebuilt == want


def _report(name, ep, ev, vmax, head, nhead):
    print("%s: per-step max position error %.2e A (step %d), velocity %.2e A/fs (%.1e of max |v|); first %d "
          "steps vs the oracle trajectory %.2e A" % (name, ep.max(), int(ep.argmax()) + 1, ev.max(),
                                                     ev.max() / vmax, nhead, head))


def test_list_mode_nve_1536_matches_oracle_and_rebuild_rule():
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["B"]
    w = water_box(8, 24.83, seed=5)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], report_interval=100, verbose=False)
    assert w["box"].min() > 2 * (6.0 + sim._neighbor_skin)  # list mode, not the lattice (image) path
    nsteps, nhead = 60, 10
    pos, vel, rebuilt, _ = run_stepwise(sim, nsteps)
    _check_rebuilds(pos, w, sim, rebuilt, 2)
    m = om.OracleModel(p, v, torch.float64, device="cuda")
    fb = oracle_force_fn(m, w["box"], w["type_idx"])
    fn = lambda r: fb(r)[0]
    mass = (w["mass"] * MU)[:, None]

    def step(r, pm, F, F1, t):
        r1, p1, _, _ = oi.vv_step(r, pm, F, mass, 0.5, lambda x: (F1, None))
        return r1, p1

    ep, ev = shadow_errors(pos, vel, mass, w["box"], fn, step)
    r, pm = w["position"].copy(), w["velocity"] * mass
    F, _ = fb(r)
    for _ in range(nhead):
        r, pm, F, _ = oi.vv_step(r, pm, F, mass, 0.5, fb)
    head = np.abs(oi.min_image_unwrap(r, pos[nhead], w["box"]) - r).max()
    vmax = np.abs(vel).max()
    _report("list-mode NVE 1,536 atoms, %d steps" % nsteps, ep, ev, vmax, head, nhead)
    assert ep.max() < 1e-5
    assert ev.max() < 5e-5 * vmax
    assert head < 1e-4


def test_config1_nvt_12288_matches_oracle():
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["A"]
    w = water_box(16, 49.66, seed=0)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.5, w["position"],
                     initial_velocity=w["velocity"], temperature=300.0, tau_t=100.0, report_interval=100,
                     verbose=False)
    nsteps, nhead = 100, 10
    pos, vel, rebuilt, chain = run_stepwise(sim, nsteps)
    _check_rebuilds(pos, w, sim, rebuilt, 1)
    m = om.OracleModel(p, v, torch.float64, device="cuda")
    fb = oracle_force_fn(m, w["box"], w["type_idx"])
    fn = lambda r: fb(r)[0]
    mass = (w["mass"] * MU)[:, None]
    kT = 300.0 * KB
    dof = 3 * len(w["type_idx"])
    xi_err, p_err = [], []

    def step(r, pm, F, F1, t):
        ch = oi.NHChain(3, dof, kT, 100.0, oi.kinetic_energy(pm, mass))
        ch.xi, ch.p = chain[t][0].copy(), chain[t][1].copy()
        r1, p1, _, _ = oi.nvt_step(r, pm, F, mass, 0.5, kT, ch, lambda x: (F1, None))
        xi_err.append(np.abs(ch.xi - chain[t + 1][0]).max())
        p_err.append(np.abs(ch.p - chain[t + 1][1]).max())
        return r1, p1

    ep, ev = shadow_errors(pos, vel, mass, w["box"], fn, step)
    r, pm = w["position"].copy(), w["velocity"] * mass
    F, _ = fb(r)
    ch = oi.NHChain(3, dof, kT, 100.0, oi.kinetic_energy(pm, mass))
    for _ in range(nhead):
        r, pm, F, _ = oi.nvt_step(r, pm, F, mass, 0.5, kT, ch, fb)
    head = np.abs(oi.min_image_unwrap(r, pos[nhead], w["box"]) - r).max()
    vmax = np.abs(vel).max()
    _report("NVT 12,288 atoms, %d steps" % nsteps, ep, ev, vmax, head, nhead)
    # chain errors against the largest |xi|, |p| the device chain reached
    xs = max(np.abs(c[0]).max() for c in chain)
    ps = max(np.abs(c[1]).max() for c in chain)
    print("chain per step: max error xi %.2e of %.2e, p %.2e of %.2e" % (max(xi_err), xs, max(p_err), ps))
    assert ep.max() < 1e-5
    assert ev.max() < 5e-5 * vmax
    assert head < 1e-4
    assert max(xi_err) < 1e-4 * xs and max(p_err) < 1e-4 * ps


def test_config3_pimd_32_beads_1536_matches_oracle_with_shared_noise():
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["B"]
    w = water_box(8, 24.83, seed=0)
    N, P, seed, nsteps = 1536, 32, 77, 2
    rng = np.random.default_rng(11)
    pos = w["position"][None] + rng.normal(scale=0.02, size=(P, N, 3))
    vel = np.broadcast_to(w["velocity"], (P, N, 3)).copy()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.25, pos,
                     initial_velocity=vel, temperature=300.0, n_bead=P, tau_t=100.0, seed=seed,
                     report_interval=10, verbose=False)
    traj = sim.run(nsteps)
    m = om.OracleModel(p, v, torch.float64, device="cuda")
    kT = 300.0 * KB
    freqs, C = oi.normal_mode_transform(P, kT)
    gamma = 2.0 * freqs
    gamma[0] = 1.0 / 100.0
    mass = (w["mass"] * MU)[:, None]
    perm = np.argsort(w["type_idx"], kind="stable")
    fb = oracle_force_fn(m, w["box"], w["type_idx"])

    def fn(R):
        return np.stack([fb(R[b])[0] for b in range(P)]), None

    R, Pm = pos.copy(), vel * mass
    F, _ = fn(R)
    for step in range(1, nsteps + 1):
        ns = philox.normals(P * N * 3, seed, step, 1).reshape(P, N, 3)
        noise = np.empty_like(ns)
        noise[:, perm] = ns                       # the device draws in type-sorted atom order
        Rn, Pm, F, _, _ = oi.pimd_step(R, Pm, F, mass, 0.25, kT, C, freqs, gamma, w["box"], noise, fn)
        R = oi.min_image_unwrap(R, Rn, w["box"])
    err = np.abs(traj["position"][-1] - R).max()
    print("PIMD 32 x 1,536, %d steps: max position error %.2e A" % (nsteps, err))
    assert err < 5e-4
