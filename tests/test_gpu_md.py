"""MD engine on the GPU (dpb_md_* through Simulation) vs the float64 oracle
integrators driven by float64 oracle forces.

Tolerances: after 20 steps of dt = 0.5 fs the FP32 device trajectory stays
within 2e-4 A (positions) and 2e-4 relative (velocities) of the FP64
oracle; Nose-Hoover chain variables within 1e-3 relative; PIMD (same
Philox noise) within 5e-4 A after 3 steps.
"""
import numpy as np
import pytest
import torch

from gpu_helpers import run_gpu
from make_golden import golden_models
from oracle import integrators as oi
from oracle import model as om
from oracle import philox

pytestmark = pytest.mark.gpu

MU = 1.036427e2
KB = 8.617333e-5


def _system():
    from deepmd_jax_b200.systems import water_box
    return water_box(4, 12.42, seed=0)


def _oracle_forces(m, w):
    def f(r):
        out = om.energy_force(m, r, w["box"], w["type_idx"], virial=False)
        return out["force"], out["energy"]
    return f


def test_nve_matches_oracle_and_conserves_energy():
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], report_interval=10, verbose=False)
    traj = sim.run(20)
    assert traj["position"].shape == (21, 192, 3)
    m = om.OracleModel(p, v, torch.float64)
    fn = _oracle_forces(m, w)
    mass = (w["mass"] * MU)[:, None]
    r, pm = w["position"].copy(), w["velocity"] * mass
    F, E0 = fn(r)
    for _ in range(20):
        r, pm, F, E = oi.vv_step(r, pm, F, mass, 0.5, fn)
    assert np.abs(traj["position"][-1] - r).max() < 2e-4
    vel = pm / mass
    assert np.abs(traj["velocity"][-1] - vel).max() < 2e-4 * np.abs(vel).max()
    # invariant drift over the run stays at the FP32 noise level
    inv = np.array([row[4] for row in sim.log])
    assert np.abs(inv - inv[0]).max() < 2e-3 * max(1.0, abs(inv[0]))


def test_nvt_nose_hoover_matches_oracle():
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.5, w["position"],
                     initial_velocity=w["velocity"], temperature=300.0, tau_t=100.0, report_interval=10,
                     verbose=False)
    traj = sim.run(20)
    r_dev = sim._report_struct()
    m = om.OracleModel(p, v, torch.float64)
    fn = _oracle_forces(m, w)
    mass = (w["mass"] * MU)[:, None]
    kT = 300.0 * KB
    r, pm = w["position"].copy(), w["velocity"] * mass
    F, _ = fn(r)
    chain = oi.NHChain(3, 3 * len(r), kT, 100.0, oi.kinetic_energy(pm, mass))
    for _ in range(20):
        r, pm, F, _ = oi.nvt_step(r, pm, F, mass, 0.5, kT, chain, fn)
    assert np.abs(traj["position"][-1] - r).max() < 2e-4
    assert np.allclose(np.array(r_dev.chain_xi[:3]), chain.xi, rtol=1e-3, atol=1e-9)
    assert np.allclose(np.array(r_dev.chain_p[:3]), chain.p, rtol=1e-3, atol=1e-7)


def test_pimd_pile_step_matches_oracle_with_shared_noise():
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    P, seed = 4, 1234
    rng = np.random.default_rng(3)
    pos = w["position"][None] + rng.normal(scale=0.02, size=(P, 192, 3))
    vel = np.broadcast_to(w["velocity"], (P, 192, 3)).copy()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.25, pos,
                     initial_velocity=vel, temperature=300.0, n_bead=P, tau_t=100.0, seed=seed,
                     report_interval=10, verbose=False)
    traj = sim.run(3)
    m = om.OracleModel(p, v, torch.float64)
    kT = 300.0 * KB
    freqs, C = oi.normal_mode_transform(P, kT)
    gamma = 2.0 * freqs
    gamma[0] = 1.0 / 100.0
    mass = (w["mass"] * MU)[:, None]
    perm = np.argsort(w["type_idx"], kind="stable")

    def fn(R):
        F = np.stack([om.energy_force(m, R[b], w["box"], w["type_idx"], virial=False)["force"] for b in range(P)])
        return F, None

    R, Pm = pos.copy(), vel * mass
    F, _ = fn(R)
    for step in range(1, 4):
        ns = philox.normals(P * 192 * 3, seed, step, 1).reshape(P, 192, 3)
        noise = np.empty_like(ns)
        noise[:, perm] = ns                       # device draws in type-sorted atom order
        Rn, Pm, F, dke, _ = oi.pimd_step(R, Pm, F, mass, 0.25, kT, C, freqs, gamma, w["box"], noise, fn)
        R = oi.min_image_unwrap(R, Rn, w["box"])
    assert np.abs(traj["position"][-1] - R).max() < 5e-4


def test_simulation_getters_and_force_match_eval():
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], verbose=False)
    ref = om.energy_force(om.OracleModel(p, v, torch.float64), w["position"], w["box"], w["type_idx"])
    assert np.abs(sim.getForce() - ref["force"]).max() <= 2e-4 * np.abs(ref["force"]).max()
    assert abs(sim.getEnergy() - ref["energy"]) < 1e-4 * max(1.0, abs(ref["energy"]))
    assert np.allclose(sim.getPosition(), w["position"], atol=1e-5)
    assert np.allclose(sim.getVelocity(), w["velocity"], rtol=1e-6, atol=1e-9)


def test_xyz_dumps_match_the_trajectory(tmp_path):
    """run(dump_prefix=...) streams every dump_interval-th frame (step 0
    included) to extended-XYZ files and returns None (md.py:907-964); the
    frames equal the in-memory trajectory of the same run."""
    from deepmd_jax_b200 import dump
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()

    def sim():
        return Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                          initial_velocity=w["velocity"], report_interval=10, type_symbols=["O", "H"],
                          verbose=False)
    traj = sim().run(20)
    prefix = str(tmp_path / "run")
    assert sim().run(20, dump_interval=5, dump_prefix=prefix, dump_content="all") is None
    fp = dump.read_xyz(prefix + "_position.xyz")
    fv = dump.read_xyz(prefix + "_velocity.xyz")
    assert [f[2].split("step=")[1].split()[0] for f in fp] == ["0", "5", "10", "15", "20"]
    for k, step in enumerate(range(0, 21, 5)):
        assert fp[k][0][:3] == [("O" if t == 0 else "H") for t in w["type_idx"][:3]]
        assert np.abs(fp[k][1] - traj["position"][step]).max() < 2e-5
        assert np.abs(fv[k][1] - traj["velocity"][step]).max() < 2e-6


def test_npt_matches_oracle_and_conserves_invariant():
    """MTK NPT with Nose-Hoover chains (deepmd_jax/routine.py:161-456) on the
    1,536-atom box, semi-isotropic couple_axes ((0, 1), (2,)): after 10 steps
    the device run and the float64 oracle agree on positions (2e-4 A), box
    lengths (2e-6 relative) and box momenta (1e-3 relative + 1e-6 abs); the
    NPT invariant of the first 30 steps stays within 1e-5 eV/atom.  (From
    step ~34 atoms of this random-weight model pass through one another and
    the invariant jumps - in NVT just the same, so the window stops before.)"""
    from deepmd_jax_b200.md import Simulation, PRESS_UNIT_CONVERSION
    from deepmd_jax_b200.systems import water_box
    from oracle import nlist as onl
    p, v = golden_models()["B"]
    w = water_box(8, 24.83, seed=3)
    N = len(w["type_idx"])
    kw = dict(temperature=300.0, pressure=1000.0, tau_t=100.0, tau_p=100.0, couple_axes=((0, 1), (2,)),
              report_interval=10, verbose=False)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.5, w["position"],
                     initial_velocity=w["velocity"], **kw)
    sim.run(10, trajectory=False)
    r_dev = sim._report_struct()
    m64 = om.OracleModel(p, v, torch.float64, device="cuda")
    cnt = np.bincount(w["type_idx"], minlength=2)

    def force_fn(r, box):
        c = onl.canonicalize(r, box, w["type_idx"])
        nb, _, _ = onl.typed_nlist(c, np.asarray(box, np.float32), onl.cutoff_sq(6.2), cnt, [80, 160])
        o = om.energy_force(m64, r, box, w["type_idx"], nbrs=nb, sel=[80, 160])
        return o["force"], (o["energy"], o["virial"])

    mass = (w["mass"] * MU)[:, None]
    kT = 300.0 * KB
    F, (E, W) = force_fn(w["position"], w["box"])
    st = oi.NPTState(w["position"], w["velocity"] * mass, F, W, mass, w["box"], 1000.0 * PRESS_UNIT_CONVERSION, kT,
                     100.0, 100.0, gid=[0, 0, 1])
    for _ in range(10):
        oi.npt_step(st, 0.5, kT, force_fn)
    assert np.abs(sim.getPosition() - st.r).max() < 2e-4
    assert np.allclose(np.array(r_dev.box), st.box(), rtol=2e-6, atol=0)
    assert np.allclose(np.array(r_dev.box_momentum[:2]), st.Pb, rtol=1e-3, atol=1e-6)
    assert r_dev.ngroups == 2
    sim.run(20, trajectory=False)
    inv = np.array([row[sim.log_headers.index("Invariant")] for row in sim.log])
    assert sim.log_headers[:5] == ["Step", "Temperature", "KE", "PE", "Pressure"]
    assert "box_x" in sim.log_headers and "box_z" in sim.log_headers
    assert len(inv) == 4 and np.abs(inv - inv[0]).max() / N < 1e-5


def test_npt_pimd_matches_oracle_with_shared_noise():
    """NPT path-integral MD (deepmd_jax/pimd.py:255-518: Parrinello-Rahman on
    the centroid mode, exact internal ring steps, PILE-L, Langevin barostat,
    centroid-virial dU/d(eps)) on the 1,536-atom box with 4 beads and
    semi-isotropic couple_axes ((0, 1), (2,)), driven by the same Philox
    noise as the float64 oracle: after 3 steps of dt = 0.25 fs positions
    agree within 5e-4 A, box lengths within 2e-6 relative, box momenta,
    dU/d(eps) and both work accumulators within 1e-3 relative."""
    from deepmd_jax_b200.md import Simulation, PRESS_UNIT_CONVERSION
    from deepmd_jax_b200.systems import water_box
    from oracle import nlist as onl
    p, v = golden_models()["B"]
    w = water_box(8, 24.83, seed=3)
    N, P, seed, tau_t, tau_p = len(w["type_idx"]), 4, 4321, 100.0, 200.0
    rng = np.random.default_rng(5)
    pos = w["position"][None] + rng.normal(scale=0.02, size=(P, N, 3))
    vel = np.broadcast_to(w["velocity"], (P, N, 3)).copy()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.25, pos,
                     initial_velocity=vel, temperature=300.0, pressure=1000.0, tau_t=tau_t, tau_p=tau_p,
                     couple_axes=((0, 1), (2,)), n_bead=P, seed=seed, report_interval=10, verbose=False)
    traj = sim.run(3)
    r_dev = sim._report_struct()
    assert int(r_dev.status) == 0
    # the trajectory carries the box of every step (md.py:784-803)
    assert traj["box"].shape == (4, 3) and np.allclose(traj["box"][0], w["box"])
    assert np.allclose(traj["box"][-1], np.array(r_dev.box), rtol=1e-6) and traj["box"][-1, 0] != traj["box"][0, 0]

    m64 = om.OracleModel(p, v, torch.float64, device="cuda")
    cnt = np.bincount(w["type_idx"], minlength=2)

    def force_fn(R, box):
        F, W = [], []
        for b in range(P):
            c = onl.canonicalize(R[b], box, w["type_idx"])
            nb, _, _ = onl.typed_nlist(c, np.asarray(box, np.float32), onl.cutoff_sq(6.2), cnt, [80, 160])
            o = om.energy_force(m64, R[b], box, w["type_idx"], nbrs=nb, sel=[80, 160])
            F.append(o["force"])
            W.append(o["virial"])
        return np.stack(F), np.stack(W)

    kT = 300.0 * KB
    freqs, C = oi.normal_mode_transform(P, kT)
    gamma = 2.0 * freqs
    gamma[0] = 1.0 / tau_t
    mass = (w["mass"] * MU)[:, None]
    perm = np.argsort(w["type_idx"], kind="stable")
    F, W = force_fn(pos, w["box"])
    st = oi.NPTPIMDState(pos, vel * mass, F, W, mass, w["box"], 1000.0 * PRESS_UNIT_CONVERSION, kT, tau_p,
                         gid=[0, 0, 1])
    for step in range(1, 4):
        ns = philox.normals(P * N * 3, seed, step, 1).reshape(P, N, 3)
        noise = np.empty_like(ns)
        noise[:, perm] = ns                       # device draws in type-sorted atom order
        nbox = philox.normals(st.G, seed, step, 2)
        prev = st.R.copy()
        oi.npt_pimd_step(st, 0.25, kT, C, freqs, gamma, 1.0 / tau_p, noise, nbox, force_fn)
        st.R = oi.min_image_unwrap(prev, st.R, st.box())
    assert np.abs(traj["position"][-1] - st.R).max() < 5e-4
    assert np.allclose(np.array(r_dev.box), st.box(), rtol=2e-6, atol=0)
    assert np.allclose(np.array(r_dev.box_momentum[:2]), st.Pb, rtol=1e-3, atol=1e-3)
    assert np.allclose(np.array(r_dev.dU_deps[:2]), st.dUde, rtol=1e-3, atol=1e-3)
    assert abs(r_dev.thermostat_work - st.twork) < 1e-3 * abs(st.twork) + 1e-4
    assert abs(r_dev.box_thermostat_work - st.btwork) < 1e-3 * abs(st.btwork) + 1e-6
    sim.run(2, trajectory=False)
    assert sim.log_headers[:5] == ["Step", "Temperature", "KE", "PE", "Pressure"]
    assert "box_x" in sim.log_headers and "box_z" in sim.log_headers


def test_autotuned_launch_shapes_leave_results_unchanged():
    """The launch-shape autotuner (dpb_md_autotune) picks candidates only and
    results do not depend on them: 12,288-atom water, mixed form, forces of
    the initial state and positions after 5 steps with and without tuning
    agree within the float-atomic summation noise (1e-5 relative, 1e-6 A)."""
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["B"]
    w = water_box(16, 49.66, seed=0)
    out = {}
    for tune in (False, True):
        sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                         initial_velocity=w["velocity"], precision="mixed", verbose=False, autotune=tune)
        if tune:
            assert sim.launch_shapes["nlist_warps_per_block"] in (4, 8, 16)
            assert sim.launch_shapes["dT_atoms_per_block"] in (2, 4, 8)
            assert sim.launch_shapes["fit_ring_stages"] in (4, 12)
        else:
            assert sim.launch_shapes is None
        F0 = sim.getForce()
        sim.run(5, trajectory=False)
        out[tune] = (F0, sim.getPosition())
    F_ref, F_tuned = out[False][0], out[True][0]
    assert np.abs(F_tuned - F_ref).max() <= 1e-5 * np.abs(F_ref).max()
    assert np.abs(out[True][1] - out[False][1]).max() < 1e-6


def test_random_velocity_com_and_pressure_getters():
    """setRandomVelocity (Maxwell-Boltzmann, centre-of-mass motion removed),
    remove_com_motion under PIMD, and getPressure from the device virial
    (deepmd_jax/md.py:744-757, 1033-1047, 1082-1090)."""
    from deepmd_jax_b200.md import Simulation, PRESS_UNIT_CONVERSION
    p, v = golden_models()["B"]
    w = _system()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.5, w["position"],
                     temperature=300.0, verbose=False)
    sim.setRandomVelocity(300.0, seed=7)
    vel = sim.getVelocity()
    m = (w["mass"] * MU)[:, None]
    assert np.abs((vel * m).sum(0)).max() < 1e-6 * np.abs(vel * m).sum()
    T = (m * vel ** 2).sum() / (3 * len(m)) / KB
    assert 200.0 < T < 400.0
    W = sim.getVirial()
    V = float(np.prod(w["box"]))
    expect = (len(m) * 300.0 * KB + np.trace(W) / 3.0) / V / PRESS_UNIT_CONVERSION
    assert abs(sim.getPressure() - expect) <= 1e-9 * max(1.0, abs(expect))
    pimd = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.25, w["position"],
                      temperature=300.0, n_bead=4, verbose=False)
    pimd.setRandomVelocity(300.0, seed=3)
    pv = pimd.getVelocity()
    assert pv.shape == (4, len(m), 3)
    assert np.abs((pv * m[None]).sum(axis=(0, 1))).max() < 1e-6 * np.abs(pv * m[None]).sum()


def test_neighbour_overflow_on_set_position_regrows_capacity():
    """Neighbour-list overflow when positions are replaced (status bit 2;
    the reference's setPosition refreshes the list and reallocates before its
    force call, md.py:985-1015, 657-668): the engine is sized on the water
    box, then set to a configuration squeezed to 70 % about the box centre
    (about 3x the neighbour density).  The capacity is re-measured, the
    forces recomputed on the full list, and the trajectory equals that of an
    engine built at the dense configuration (float-atomic noise only)."""
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    c = w["box"] / 2
    dense = c + 0.7 * (w["position"] - c)
    kw = dict(initial_velocity=w["velocity"], report_interval=10, verbose=False, autotune=False)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.25, w["position"], **kw)
    sel0 = list(sim._sel)
    sim.setPosition(dense)
    sim.setVelocity(w["velocity"])
    sim.run(5, trajectory=False)
    assert int(sim._report_struct().status) == 0
    assert all(a > b for a, b in zip(sim._sel, sel0))      # the capacity grew
    ref = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.25, dense, **kw)
    ref.run(5, trajectory=False)
    assert list(ref._sel) == list(sim._sel)
    assert np.abs(sim.getPosition() - ref.getPosition()).max() < 1e-5


def test_nve_with_com_motion_removed_matches_oracle():
    """remove_com_motion=True (md.py:793-796): after every step the
    centre-of-mass velocity is subtracted (v <- v - sum(m v) / sum(m)).
    Initial velocities with a drift of 1e-3 A/fs; after 10 steps positions
    and velocities match the float64 oracle doing the same, and the total
    momentum is zero to float32 precision."""
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    vel0 = w["velocity"] + np.array([1e-3, -2e-3, 5e-4])
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=vel0, remove_com_motion=True, report_interval=10, verbose=False)
    traj = sim.run(10)
    m = om.OracleModel(p, v, torch.float64)
    fn = _oracle_forces(m, w)
    mass = (w["mass"] * MU)[:, None]
    r, pm = w["position"].copy(), vel0 * mass
    F, _ = fn(r)
    for _ in range(10):
        r, pm, F, _ = oi.vv_step(r, pm, F, mass, 0.5, fn)
        pm = pm - mass * pm.sum(0) / mass.sum()
    assert np.abs(traj["position"][-1] - r).max() < 2e-4
    vel = pm / mass
    assert np.abs(traj["velocity"][-1] - vel).max() < 2e-4 * np.abs(vel).max()
    P = (traj["velocity"][-1] * mass).sum(0)
    assert np.abs(P).max() < 1e-5 * np.abs(traj["velocity"][-1] * mass).sum()


def test_fixed_atoms_nvt_with_com_removal_and_nve_match_oracle():
    """fixed_indices (md.py:221-236, routine.py:110-136): fixed atoms never
    move (bitwise), their forces read zero (md.py:428-430), the chain has
    3 n_mobile degrees of freedom, the temperature is scaled by
    N / n_mobile (md.py:478), and the centre-of-mass velocity comes from the
    mobile atoms only while it is subtracted from every atom (md.py:788-789).
    NVT with remove_com_motion for 10 steps and NVE for 10 steps against the
    float64 oracle; the NVT report's KE is that of the final (scaled)
    momenta."""
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    N = len(w["type_idx"])
    fixed = np.array(sorted(set(range(0, N, 7)) | set(range(40, 52))))
    mob = np.ones(N, dtype=bool)
    mob[fixed] = False
    m = om.OracleModel(p, v, torch.float64)
    fn = oi.fixed_atom_forces(_oracle_forces(m, w), mob)
    mass = (w["mass"] * MU)[:, None]
    kT = 300.0 * KB
    vel0 = w["velocity"] + np.array([1e-3, -2e-3, 5e-4])

    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.5, w["position"],
                     initial_velocity=vel0, temperature=300.0, tau_t=100.0, remove_com_motion=True,
                     fixed_indices=list(fixed), report_interval=10, verbose=False)
    pos32 = w["position"].astype(np.float32).astype(np.float64)
    assert np.all(sim.getForce()[fixed] == 0.0) and np.all(sim.getVelocity()[fixed] == 0.0)
    traj = sim.run(10)
    r_dev = sim._report_struct()
    assert r_dev.chain_dof == 3 * mob.sum()
    r, pm = w["position"].copy(), oi.mask_momenta(vel0 * mass, mob)
    F, _ = fn(r)
    chain = oi.NHChain(3, 3 * int(mob.sum()), kT, 100.0, oi.kinetic_energy(pm, mass))
    for _ in range(10):
        r, pm, F, _ = oi.nvt_step(r, pm, F, mass, 0.5, kT, chain, fn, mob)
        V = (pm * mob[:, None]).sum(0) / (mass[:, 0] * mob).sum()
        pm = pm - mass * V
    assert np.array_equal(traj["position"][:, fixed], np.broadcast_to(pos32[fixed], traj["position"][:, fixed].shape))
    assert np.abs(traj["position"][-1] - r).max() < 2e-4
    vel = pm / mass
    assert np.abs(traj["velocity"][-1] - vel).max() < 2e-4 * np.abs(vel).max()
    assert np.allclose(np.array(r_dev.chain_xi[:3]), chain.xi, rtol=1e-3, atol=1e-9)
    assert np.allclose(np.array(r_dev.chain_p[:3]), chain.p, rtol=1e-3, atol=1e-7)
    assert np.all(sim.getForce()[fixed] == 0.0)
    ke = oi.kinetic_energy(pm, mass)
    assert abs(sim.log[-1][2] - ke) <= 1e-4 * ke
    assert abs(sim.log[-1][1] - 2 * ke / (3 * mob.sum()) / KB) <= 1e-4 * sim.log[-1][1]

    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE", 0.5, w["position"],
                     initial_velocity=w["velocity"], fixed_indices=list(fixed), report_interval=10, verbose=False)
    traj = sim.run(10)
    r, pm = w["position"].copy(), oi.mask_momenta(w["velocity"] * mass, mob)
    F, _ = fn(r)
    for _ in range(10):
        r, pm, F, _ = oi.vv_step(r, pm, F, mass, 0.5, fn, mob)
        pm = oi.mask_momenta(pm, mob)
    assert np.array_equal(traj["position"][-1][fixed], pos32[fixed])
    assert np.all(traj["velocity"][-1][fixed] == 0.0)
    assert np.abs(traj["position"][-1] - r).max() < 2e-4
    assert np.abs(traj["velocity"][-1] - pm / mass).max() < 2e-4 * np.abs(pm / mass).max()
    with pytest.raises(NotImplementedError):
        Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NPT", 0.5, w["position"],
                   temperature=300.0, pressure=1.0, fixed_indices=[0], verbose=False)


def test_model_deviation_reporter_matches_separate_evaluations():
    """model_deviation_paths (md.py:299-302,559-567): at each report the
    forces of every deviation model on the current positions and neighbour
    list; Model_Devi = max over atoms and axes of their standard deviation
    over models.  Checked against separate FP32 evaluations of the three
    models on the final positions (relative 1e-4)."""
    from deepmd_jax_b200.md import Simulation
    from make_golden import hermite_compressed
    models = golden_models()
    p, v = models["B"]
    devs = [models["B"], models["A"], hermite_compressed(*models["B"])]
    w = _system()
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.5, w["position"],
                     initial_velocity=w["velocity"], temperature=300.0, model_deviation_paths=devs,
                     report_interval=10, verbose=False)
    sim.run(10)
    assert sim.log_headers[-2] == "Model_Devi"
    pos = sim.getPosition()
    F = np.stack([run_gpu(dp, dv, pos, w["box"], w["type_idx"])["force"][0] for dp, dv in devs])
    want = F.std(axis=0).max()
    assert abs(sim.log[-1][-2] - want) <= 1e-4 * want
    assert abs(sim.model_deviation() - sim.log[-1][-2]) <= 1e-5 * want  # float atomics: last bits may differ
    with pytest.raises(NotImplementedError):
        Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.5, w["position"],
                   temperature=300.0, n_bead=2, model_deviation_paths=devs[:1], verbose=False)


def test_langevin_matches_oracle_with_shared_noise():
    """routine='NVT_langevin' (routine.py:46-107, md.py:352-356): BAOAB with
    friction 1/tau_t, noise from the same Philox stream (tag 3) in the
    oracle; 10 steps with fixed atoms and centre-of-mass removal (the
    Langevin step keeps the fixed atoms' momenta, md.py:788-789); positions,
    velocities and the thermostat work against the float64 oracle, and the
    Invariant KE + PE - work reported."""
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    N = len(w["type_idx"])
    fixed = np.arange(0, N, 9)
    mob = np.ones(N, dtype=bool)
    mob[fixed] = False
    seed = 11
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT_langevin", 0.5, w["position"],
                     initial_velocity=w["velocity"], temperature=300.0, tau_t=50.0, seed=seed,
                     fixed_indices=list(fixed), remove_com_motion=True, report_interval=10, verbose=False)
    traj = sim.run(10)
    assert sim.log_headers[:5] == ["Step", "Temperature", "KE", "PE", "Invariant"]
    r_dev = sim._report_struct()
    m = om.OracleModel(p, v, torch.float64)
    fn = oi.fixed_atom_forces(_oracle_forces(m, w), mob)
    mass = (w["mass"] * MU)[:, None]
    kT = 300.0 * KB
    perm = np.argsort(w["type_idx"], kind="stable")
    r, pm = w["position"].copy(), oi.mask_momenta(w["velocity"] * mass, mob)
    F, _ = fn(r)
    work = 0.0
    for step in range(1, 11):
        ns = philox.normals(N * 3, seed, step, 3).reshape(N, 3)
        noise = np.empty_like(ns)
        noise[perm] = ns                          # device draws in type-sorted atom order
        r, pm, F, _, dW = oi.langevin_step(r, pm, F, mass, 0.5, kT, 1.0 / 50.0, noise, fn, mob)
        work += dW
        V = (pm * mob[:, None]).sum(0) / (mass[:, 0] * mob).sum()
        pm = pm - mass * V
    assert np.abs(traj["position"][-1] - r).max() < 2e-4
    vel = pm / mass
    assert np.abs(traj["velocity"][-1] - vel).max() < 2e-4 * np.abs(vel).max()
    assert abs(r_dev.thermostat_work - work) <= 2e-3 * abs(work) + 1e-4
    ke = oi.kinetic_energy(pm, mass)
    assert abs(sim.log[-1][4] - (sim.log[-1][2] + sim.log[-1][3] - r_dev.thermostat_work)) <= 1e-9
    assert abs(sim.log[-1][2] - ke) <= 1e-4 * ke


def test_pimd_invariant_reporter_matches_state():
    """pimd_print_invariant (md.py:512-521): Invariant = (KE + sum of bead
    energies + spring energy - thermostat work) / P, recomputed from the
    returned final state with float64 oracle energies and the oracle's
    unwrap across beads (relative 1e-5)."""
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    P = 4
    rng = np.random.default_rng(5)
    pos = w["position"][None] + rng.normal(scale=0.02, size=(P, 192, 3))
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVT", 0.25, pos,
                     temperature=300.0, n_bead=P, tau_t=100.0, seed=7, pimd_print_invariant=True,
                     report_interval=10, verbose=False)
    traj = sim.run(10)
    assert sim.log_headers[4] == "Invariant"
    r_dev = sim._report_struct()
    m = om.OracleModel(p, v, torch.float64)
    R, V = traj["position"][-1], traj["velocity"][-1]
    mass = (w["mass"] * MU)[:, None]
    E = sum(om.energy_force(m, R[b], w["box"], w["type_idx"], virial=False)["energy"] for b in range(P))
    KE = 0.5 * float((mass * V ** 2).sum())
    Ru = oi.unwrap_across_beads(R, w["box"])
    omega = P * 300.0 * KB / oi.HBAR
    spring = 0.5 * omega ** 2 * float((mass * (Ru - np.roll(Ru, 1, axis=0)) ** 2).sum())
    want = (KE + E + spring - r_dev.thermostat_work) / P
    scale = (abs(E) + KE + spring) / P
    assert abs(sim.log[-1][4] - want) <= 1e-5 * scale, (sim.log[-1][4], want)


@pytest.mark.parametrize("n_bead", [1, 3])
def test_trajectory_frames_kernel_matches_host_unpermute(n_bead):
    """dpb_md_traj_frames (type-sorted float32 frames -> user-order float64
    positions and velocities) against the host's un-permute and float64
    division (Simulation._unpack_frame), bit for bit, on random frames; then
    a two-chunk run() whose last trajectory frame is the engine's own state."""
    from deepmd_jax_b200.md import Simulation
    p, v = golden_models()["B"]
    w = _system()
    if n_bead == 1:
        pos, vel, kw = w["position"], w["velocity"], {}
    else:
        pos = np.broadcast_to(w["position"], (n_bead, 192, 3)).copy()
        vel = np.broadcast_to(w["velocity"], (n_bead, 192, 3)).copy()
        kw = dict(temperature=300.0, n_bead=n_bead, tau_t=100.0, seed=5)
    sim = Simulation((p, v), w["box"], w["type_idx"], w["mass_per_type"], "NVE" if n_bead == 1 else "NVT",
                     0.25, pos, initial_velocity=vel, report_interval=10, verbose=False, **kw)
    n, nf3 = 5, n_bead * 192 * 3
    g = torch.Generator(device="cuda").manual_seed(0)
    bp = torch.randn((n, nf3), device="cuda", generator=g) * 20.0
    bv = torch.randn((n, nf3), device="cuda", generator=g)
    op = torch.full((n, nf3), np.nan, dtype=torch.float64, device="cuda")
    ov = torch.full((n, nf3), np.nan, dtype=torch.float64, device="cuda")
    rc = sim.lib.dpb_md_traj_frames(sim._h, n, bp.data_ptr(), bv.data_ptr(), op.data_ptr(), ov.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0
    for i in range(n):
        ep, ev = sim._unpack_frame(bp[i], bv[i])
        assert np.array_equal(op[i].cpu().numpy().reshape(ep.shape), ep)
        assert np.array_equal(ov[i].cpu().numpy().reshape(ev.shape), ev)
    traj = sim.run(12)   # chunks of 10 and 2 steps: both frame buffers
    assert traj["position"].shape[0] == 13
    assert np.array_equal(traj["position"][-1], sim.getPosition())
    assert np.allclose(traj["velocity"][-1], sim.getVelocity(), rtol=1e-6, atol=1e-12)
