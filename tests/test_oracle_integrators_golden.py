"""The oracle's integrators against golden steps of the reference's own
integrator source (tests/golden/golden_integrators.npz, written by
tests/golden/make_golden_integrators.py from deepmd_jax/pimd.py and
deepmd_jax/routine.py): one NVT ring-polymer BAOAB step with PILE-L, one
NPT ring-polymer step with the Langevin barostat (axes x, y coupled, z
alone), one classical BAOAB Langevin step with fixed atoms and three MTK
NPT steps, each on a Gaussian pair potential with the saved noise.  float64
on both sides: agreement to 1e-9 relative."""
import os

import numpy as np
import torch

from oracle import integrators as oi

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_integrators.npz"))
A, S2 = G["pair"]
BOX = G["box"]


def _bead_energies(R, box, eps=None):
    """Per-bead Gaussian pair energies of R (P, N, 3), optionally strained by
    (1 + eps) per axis (coordinates and box together)."""
    R = torch.as_tensor(R)
    scale = 1.0 if eps is None else 1.0 + eps
    L = torch.as_tensor(box) * scale
    X = R * scale
    d = X[:, :, None, :] - X[:, None, :, :]
    d = d - L * torch.round(d / L)
    r2 = (d * d).sum(-1)
    off = ~torch.eye(R.shape[1], dtype=torch.bool)
    return 0.5 * (A * torch.exp(-r2 / S2))[:, off].sum(-1)


def _forces(R, box):
    x = torch.tensor(R, dtype=torch.float64, requires_grad=True)
    return -torch.autograd.grad(_bead_energies(x, box).sum(), x)[0].numpy()


def _forces_and_virials(R, box):
    """Forces and per-bead virials W_b with W_b,aa = -dE_b / d eps_a."""
    W = np.zeros((R.shape[0], 3, 3))
    for b in range(R.shape[0]):
        eps = torch.zeros(3, dtype=torch.float64, requires_grad=True)
        g = torch.autograd.grad(_bead_energies(R[b:b + 1], box, eps).sum(), eps)[0].numpy()
        W[b] = -np.diag(g)
    return _forces(R, box), W


def _close(got, want, name, rtol=1e-9):
    scale = max(np.abs(want).max(), 1e-12)
    assert np.abs(np.asarray(got) - want).max() <= rtol * scale, (name, np.abs(np.asarray(got) - want).max(), scale)


def test_nvt_ring_polymer_step_matches_reference():
    m = G["mass"]
    F0 = _forces(G["R0"], BOX)
    R, P, F, dke, _ = oi.pimd_step(G["R0"].copy(), G["P0"].copy(), F0, m, float(G["dt"]), float(G["kT"]), G["C"],
                                   G["freqs"], G["gamma"], BOX, G["nvt_noise"], lambda r: (_forces(r, BOX), None))
    _close(R, G["nvt_R"], "R")
    _close(P, G["nvt_P"], "P")
    _close(F, G["nvt_F"], "F")
    _close(dke, G["nvt_work"], "work")


def test_npt_ring_polymer_step_matches_reference():
    m, kT, dt = G["mass"], float(G["kT"]), float(G["dt"])
    tau_p = float(G["npt_tau_p"])
    F0, W0 = _forces_and_virials(G["R0"], BOX)
    st = oi.NPTPIMDState(G["R0"], G["P0"], F0, W0, m, BOX, float(G["npt_pressure"]), kT, tau_p, G["npt_gid"])
    _close(st.Mb, G["npt_Mb"], "box mass")
    _close(st.dUde, G["npt_dUdV0"], "dU/deps at init")
    st.Pb = G["npt_Pb0"].copy()
    oi.npt_pimd_step(st, dt, kT, G["C"], G["freqs"], G["gamma"], 1.0 / tau_p, G["npt_noise"], G["npt_noise_b"],
                     _forces_and_virials)
    _close(st.R, G["npt_R"], "R")
    _close(st.P, G["npt_P"], "P")
    _close(st.F, G["npt_F"], "F")
    _close(st.Rb, G["npt_Rb"], "box position")
    _close(st.Pb, G["npt_Pb"], "box momentum")
    _close(st.dUde, G["npt_dUdV"], "dU/deps")
    _close(st.twork, G["npt_work"], "work")
    _close(st.btwork, G["npt_box_work"], "box work")


def test_langevin_step_with_fixed_atoms_matches_reference():
    m, mob = G["mass"], G["lan_mobile"]
    fn = oi.fixed_atom_forces(lambda r: (_forces(r[None], BOX)[0], None), mob)
    F0, _ = fn(G["lan_r0"])
    r, p, F, _, dW = oi.langevin_step(G["lan_r0"].copy(), G["lan_p0"].copy(), F0, m, float(G["dt"]),
                                      float(G["kT"]), 1.0 / 50.0, G["lan_noise"], fn, mob)
    _close(r, G["lan_R"], "R")
    _close(p, G["lan_P"], "P")
    _close(F, G["lan_F"], "F")
    _close(dW, G["lan_work"], "work")
    assert np.array_equal(r[~mob], G["lan_r0"][~mob]) and np.all(p[~mob] == 0.0)


def test_mtk_npt_steps_match_reference():
    """Three MTK NPT steps with Nose-Hoover thermostat and barostat chains,
    axis x alone and y, z coupled (routine.py:230-426).  The chain substep
    of the fixture is the oracle's restatement of jax_md's (jax_md is
    absent), so this pins the barostat, the coupled axes and the step order."""
    m, kT, dt = G["mass"], float(G["kT"]), float(G["dt"])
    r0 = G["R0"][0]
    p0 = G["P0"][0] / np.sqrt(float(G["P"]))

    def force_fn(r, box):
        F, W = _forces_and_virials(r[None], box)
        return F[0], (float(_bead_energies(r[None], box)[0]), W[0])

    F0, (_, W0) = force_fn(r0, BOX)
    st = oi.NPTState(r0, p0, F0, W0, m, BOX, float(G["mtk_pressure"]), kT, float(G["mtk_tau_t"]),
                     float(G["mtk_tau_p"]), G["mtk_gid"])
    _close(st.dUde, G["mtk_dUdV0"], "dU/deps at init")
    st.Pb = G["mtk_Pb0"].copy()
    for _ in range(3):
        oi.npt_step(st, dt, kT, force_fn)
    _close(st.r, G["mtk_R"], "R")
    _close(st.p, G["mtk_P"], "P")
    _close(st.F, G["mtk_F"], "F")
    _close(st.Rb, G["mtk_Rb"], "box position")
    _close(st.Pb, G["mtk_Pb"], "box momentum")
    _close(st.dUde, G["mtk_dUdV"], "dU/deps")
    _close(st.thermo.xi, G["mtk_xi"], "thermostat xi")
    _close(st.thermo.p, G["mtk_pxi"], "thermostat p")
    _close(st.baro.xi, G["mtk_bxi"], "barostat xi")
    _close(st.baro.p, G["mtk_bpxi"], "barostat p")


def test_fixed_atom_wrapper_nve_and_nvt_match_reference():
    """with_fixed_atoms around NVE and Nose-Hoover NVT (routine.py:110-158),
    three steps each: momenta masked at init and after every step, fixed
    coordinates under stop_gradient, the masked shift of md.py:231-234, and
    for NVT the chain over 3 n_mobile degrees of freedom with
    Q0 = kT tau^2 DOF and the initial kinetic energy of the masked momenta.
    jax_md's own NVE / NVT steps are restated in the fixture, so this pins
    the wrapper."""
    m, mob, kT, dt = G["mass"], G["lan_mobile"], float(G["kT"]), float(G["dt"])
    fn = oi.fixed_atom_forces(lambda r: (_forces(r[None], BOX)[0], None), mob)
    r0 = G["lan_r0"]
    # NVE
    p = G["fnve_p0"].copy()
    assert np.all(p[~mob] == 0.0)
    r, (F, _) = r0.copy(), fn(r0)
    for _ in range(3):
        r, p, F, _ = oi.vv_step(r, p, F, m, dt, fn, mob)
        p = oi.mask_momenta(p, mob)
    _close(r, G["fnve_R"], "NVE R")
    _close(p, G["fnve_P"], "NVE P")
    # NVT
    p = G["fnvt_p0"].copy()
    chain = oi.NHChain(3, 3 * int(mob.sum()), kT, 60.0, oi.kinetic_energy(p, m))
    _close(chain.Q, G["fnvt_Q0"], "chain masses at init")
    _close(chain.KE, G["fnvt_KE0"], "chain KE at init")
    r, (F, _) = r0.copy(), fn(r0)
    for _ in range(3):
        r, p, F, _ = oi.nvt_step(r, p, F, m, dt, kT, chain, fn, mob)
    _close(r, G["fnvt_R"], "NVT R")
    _close(p, G["fnvt_P"], "NVT P")
    _close(chain.xi, G["fnvt_xi"], "chain xi")
    _close(chain.p, G["fnvt_pxi"], "chain p")
