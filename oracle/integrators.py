"""ORACLE (test infrastructure only): float64 restatement of the MD updates
on the reference's hot path.

  * velocity Verlet (jax_md.simulate.nve / velocity_verlet, wrapped by
    deepmd_jax/routine.py:139-144);
  * Martyna-Tuckerman-Klein Nose-Hoover chain (jax_md.simulate.nvt_nose_hoover
    and nose_hoover_chain, wrapped by deepmd_jax/routine.py:147-158), chain
    masses Q = kT tau^2 (Q0 *= DOF), DOF = 3N (3 n_mobile with fixed atoms,
    deepmd_jax/routine.py:110-136); invariant per deepmd_jax/routine.py:9-25;
  * BAOAB Langevin with the thermostat work (deepmd_jax/routine.py:46-107);
  * PIMD BAOAB with exact free ring-polymer propagation and the PILE-L
    thermostat (deepmd_jax/pimd.py:22-44,92-111,114-207,210-247);
  * MTK NPT with Nose-Hoover chains on the particles and on the box, axes in
    coupled groups (deepmd_jax/routine.py:161-456);
  * NPT-PIMD: Parrinello-Rahman on the centroid mode, exact internal ring
    steps, PILE-L and a Langevin barostat, centroid-virial strain
    derivative (deepmd_jax/pimd.py:255-518);
  * min_image_unwrap (deepmd_jax/md_utils.py:162-169).

jax_md is a third-party dependency that is absent here (unpinned git HEAD,
setup.py:13); the Nose-Hoover substep below restates its published MTK
algorithm (Martyna, Tuckerman, Tobias, Klein, Mol. Phys. 87, 1117 (1996)) with
the operator order used by jax_md.  Parity of that order is unpinned.
The ring-polymer steps (NVT and NPT), the BAOAB Langevin step, the MTK NPT
step (all but its chain substep) and the fixed-atom wrapper of NVE / NVT
are pinned to the reference's own source by
tests/test_oracle_integrators_golden.py.
The Gaussian noise of the stochastic steps comes from oracle/philox.py, the
same counter-based stream the device kernels draw, so a step can be compared
deterministically.
"""
from __future__ import annotations

import numpy as np

HBAR = 6.582119569e-16 * 1e15  # eV fs (deepmd_jax/pimd.py:19)


def kinetic_energy(p, m):
    return 0.5 * float((p * p / m).sum())


def vv_step(r, p, F, m, dt, force_fn, mobile=None):
    """One velocity-Verlet step; returns (r, p, F, extra) with extra from force_fn.
    mobile (N,) bool: fixed atoms keep their positions (the masked shift of
    deepmd_jax/md.py:231-234); force_fn must then be fixed_atom_forces(...)
    and the caller masks the momenta after the step (mask_momenta)."""
    p = p + 0.5 * dt * F
    dr = dt * p / m
    r = r + (dr if mobile is None else dr * mobile[:, None])
    F, extra = force_fn(r)
    p = p + 0.5 * dt * F
    return r, p, F, extra


def mask_momenta(p, mobile):
    """with_fixed_atoms (deepmd_jax/routine.py:130-134): the fixed atoms'
    momenta are zeroed after every step of the wrapped integrator."""
    return p if mobile is None else p * mobile[:, None]


def fixed_atom_forces(force_fn, mobile):
    """Forces with the fixed atoms' coordinates under stop_gradient
    (deepmd_jax/md.py:428-430): their rows are zero, the mobile rows keep
    every term."""
    def f(r):
        F, extra = force_fn(r)
        return F * mobile[:, None], extra
    return f


class NHChain:
    """Nose-Hoover chain state (float64)."""

    def __init__(self, chain_length, dof, kT, tau, KE):
        self.L = chain_length
        self.xi = np.zeros(chain_length)
        self.p = np.zeros(chain_length)
        self.Q = kT * tau ** 2 * np.ones(chain_length)
        self.Q[0] *= dof
        self.dof = dof
        self.tau = tau
        self.KE = KE

    def update_mass(self, kT):
        self.Q = kT * self.tau ** 2 * np.ones(self.L)
        self.Q[0] *= self.dof

    def substep(self, delta, P, kT):
        """One MTK chain substep of length delta/2 (jax_md nose_hoover_chain)."""
        d2, d4, d8 = delta / 2, delta / 4, delta / 8
        p, Q = self.p.copy(), self.Q
        M = self.L - 1
        G = p[M - 1] ** 2 / Q[M - 1] - kT
        p[M] += d4 * G
        for m in range(M - 1, 0, -1):
            G = p[m - 1] ** 2 / Q[m - 1] - kT
            scale = np.exp(-d8 * p[m + 1] / Q[m + 1])
            p[m] = scale * (scale * p[m] + d4 * G)
        G = 2.0 * self.KE - self.dof * kT
        scale = np.exp(-d8 * p[1] / Q[1])
        p[0] = scale * (scale * p[0] + d4 * G)
        scale = np.exp(-d2 * p[0] / Q[0])
        self.KE = self.KE * scale ** 2
        P = P * scale
        self.xi = self.xi + d2 * p / Q
        G = 2.0 * self.KE - self.dof * kT
        for m in range(M):
            scale = np.exp(-d8 * p[m + 1] / Q[m + 1])
            p[m] = scale * (scale * p[m] + d4 * G)
            G = p[m] ** 2 / Q[m] - kT
        p[M] += d4 * G
        self.p = p
        return P

    def invariant_terms(self, kT):
        """Chain part of the NH invariant (deepmd_jax/routine.py:19-24)."""
        E = self.p[0] ** 2 / (2 * self.Q[0]) + self.dof * kT * self.xi[0]
        for r, p, q in zip(self.xi[1:], self.p[1:], self.Q[1:]):
            E += p ** 2 / (2 * q) + kT * r
        return E


def nvt_step(r, p, F, m, dt, kT, chain: NHChain, force_fn, mobile=None):
    """One Nose-Hoover NVT step; with mobile, the chain's dof must be
    3 n_mobile (deepmd_jax/routine.py:115-132) and the momenta are masked
    after the step."""
    chain.update_mass(kT)
    p = chain.substep(dt, p, kT)
    r, p, F, extra = vv_step(r, p, F, m, dt, force_fn, mobile)
    chain.KE = kinetic_energy(p, m)
    p = chain.substep(dt, p, kT)
    return r, mask_momenta(p, mobile), F, extra


def langevin_step(r, p, F, m, dt, kT, gamma, noise, force_fn, mobile=None):
    """One BAOAB Langevin step (deepmd_jax/routine.py:81-103): B, A, O with
    c1 = exp(-gamma dt), c2 = sqrt(kT (1 - c1^2)) and the noise zeroed on
    fixed atoms, A, force, B.  Returns (r, p, F, extra, dW) with dW the
    kinetic-energy change of the O step (the thermostat work)."""
    mob = None if mobile is None else mobile[:, None]
    p = p + 0.5 * dt * F
    r = r + 0.5 * dt * p / m * (1 if mob is None else mob)
    c1 = np.exp(-gamma * dt)
    c2 = np.sqrt(max(kT * (1.0 - c1 ** 2), 0.0))
    xi = noise if mob is None else noise * mob
    pn = c1 * p + c2 * np.sqrt(m) * xi
    dW = 0.5 * float(((pn ** 2 - p ** 2) / m).sum())
    r = r + 0.5 * dt * pn / m * (1 if mob is None else mob)
    F, extra = force_fn(r)
    pn = pn + 0.5 * dt * F
    return r, pn, F, extra, dW


def sinhx_x(x):
    """sinh(x)/x by the series of deepmd_jax/routine.py:290-292."""
    return 1 + x ** 2 / 6 + x ** 4 / 120 + x ** 6 / 5040 + x ** 8 / 362_880 + x ** 10 / 39_916_800


class NPTState:
    """MTK NPT state with coupled axis groups (deepmd_jax/routine.py:161-456):
    log box scales Rb, momenta Pb, masses Mb per group, the cached per-group
    dU/d(eps), a thermostat chain (DOF 3N, tau_t) and a barostat chain (DOF G,
    tau_p).  force_fn(r, box) -> (F, (E, W)) with W the virial, whose
    diagonal gives dU/d(eps_a) = -W_aa."""

    def __init__(self, r, p, F, W, m, box, pressure, kT, tau_t, tau_p, gid, chain_t=3, chain_p=3):
        self.r, self.p, self.F, self.m = r.copy(), p.copy(), F.copy(), m
        self.ref = np.asarray(box, float).copy()
        self.gid = np.asarray(gid)
        self.G = int(self.gid.max()) + 1
        self.ngrp = np.array([(self.gid == g).sum() for g in range(self.G)], float)
        N = r.shape[0]
        self.Rb = np.zeros(self.G)
        self.Pb = np.zeros(self.G)
        self.tau_p = tau_p
        self.Mb = self.ngrp * (N + 1) * kT * tau_p ** 2
        self.dUde = self.dU_deps(W)
        self.pressure = pressure
        self.thermo = NHChain(chain_t, 3 * N, kT, tau_t, kinetic_energy(p, m))
        self.baro = NHChain(chain_p, self.G, kT, tau_p, 0.0)

    def dU_deps(self, W):
        out = np.zeros(self.G)
        for a in range(3):
            if self.gid[a] >= 0:
                out[self.gid[a]] -= W[a, a]
        return out

    def box(self):
        return self.ref * np.array([np.exp(self.Rb[g]) if g >= 0 else 1.0 for g in self.gid])

    def box_force(self, V, Nf):
        KE2 = (self.p ** 2 / self.m).sum(0)
        tot = KE2.sum()
        grp = np.array([KE2[self.gid == g].sum() for g in range(self.G)])
        return grp + (self.ngrp / Nf) * tot - self.dUde - self.pressure * V * self.ngrp


def npt_step(st: NPTState, dt, kT, force_fn):
    """One apply_fn step of npt_nose_hoover (deepmd_jax/routine.py:403-436)."""
    N = st.r.shape[0]
    Nf = 3.0 * N
    st.thermo.update_mass(kT)
    st.baro.update_mass(kT)
    st.Mb = st.ngrp * (N + 1) * kT * st.tau_p ** 2
    st.Pb = st.baro.substep(dt, st.Pb, kT)
    st.p = st.thermo.substep(dt, st.p, kT)
    # inner step
    G = st.box_force(np.prod(st.box()), Nf)
    st.Pb = st.Pb + 0.5 * dt * G
    Vb = st.Pb / st.Mb
    va = np.array([Vb[g] if g >= 0 else 0.0 for g in st.gid])
    rate = va + (st.ngrp * Vb).sum() / Nf
    x = rate * dt / 2

    def exp_iL2(p, F):
        return p * np.exp(-x) + (dt / 2) * F * sinhx_x(x / 2) * np.exp(-x / 2)

    st.p = exp_iL2(st.p, st.F)
    st.Rb = st.Rb + Vb * dt
    box = st.box()
    y = va * dt
    st.r = st.r * np.exp(y) + dt * (st.p / st.m) * np.exp(y / 2) * sinhx_x(y / 2)
    F, (E, W) = force_fn(st.r, box)
    st.F = F
    st.dUde = st.dU_deps(W)
    st.p = exp_iL2(st.p, F)
    G = st.box_force(np.prod(box), Nf)
    st.Pb = st.Pb + 0.5 * dt * G
    st.thermo.KE = kinetic_energy(st.p, st.m)
    st.baro.KE = 0.5 * float((st.Pb ** 2 / st.Mb).sum())
    st.p = st.thermo.substep(dt, st.p, kT)
    st.Pb = st.baro.substep(dt, st.Pb, kT)
    return E, W


def normal_mode_transform(n_bead, kT):
    """(freqs (P,), C (P,P)) exactly as deepmd_jax/pimd.py:22-44 (numpy eigh)."""
    ring_poly_freq = n_bead * kT / HBAR
    A = (2 * np.eye(n_bead) - np.roll(np.eye(n_bead), 1, axis=0) - np.roll(np.eye(n_bead), -1, axis=0))
    eva, eve = np.linalg.eigh(A)
    order = np.argsort(eva)
    eva = eva[order]
    eve = eve[:, order]
    if n_bead >= 2:
        eva[0] = 0.0
    return ring_poly_freq * np.sqrt(np.maximum(eva, 0.0)), eve


def unwrap_across_beads(R, box3):
    ref = R[0:1]
    d = R - ref
    d = d - box3 * np.round(d / box3)
    return ref + d


def free_ring_step(R, P, m, C, w, h, box3):
    """Exact free ring-polymer propagation for time h (pimd.py:160-179).
    R, P: (P, N, 3); m: (N, 1)."""
    R = unwrap_across_beads(R, box3)
    Q = np.tensordot(C.T, R, axes=(1, 0))
    Pn = np.tensordot(C.T, P, axes=(1, 0))
    w = w[:, None, None]
    c, s = np.cos(w * h), np.sin(w * h)
    sw = np.where(w == 0, 1.0, w)
    Qn = np.empty_like(Q)
    Pm = np.empty_like(Pn)
    Qn[0] = Q[0] + h * Pn[0] / m
    Pm[0] = Pn[0]
    Qn[1:] = Q[1:] * c[1:] + Pn[1:] * s[1:] / (m * sw[1:])
    Pm[1:] = Pn[1:] * c[1:] - m * sw[1:] * Q[1:] * s[1:]
    return np.tensordot(C, Qn, axes=(1, 0)), np.tensordot(C, Pm, axes=(1, 0))


def pile_l_step(P, m, C, gamma, dt, kT, noise):
    """PILE-L O step in normal modes (pimd.py:92-111); noise (P, N, 3) ~ N(0,1).
    Returns (P_new, delta_KE)."""
    nb = C.shape[0]
    Pn = np.tensordot(C.T, P, axes=(1, 0))
    c1 = np.exp(-gamma * dt)[:, None, None]
    c2 = np.sqrt(np.maximum(kT * nb * (1.0 - c1 ** 2), 0.0))
    Pn = c1 * Pn + c2 * np.sqrt(m) * noise
    Pnew = np.tensordot(C, Pn, axes=(1, 0))
    dKE = 0.5 * float(((Pnew ** 2 - P ** 2) / m).sum())
    return Pnew, dKE


def pimd_step(R, P, F, m, dt, kT, C, w, gamma, box3, noise, force_fn):
    """One BAOAB PIMD step (pimd.py:193-205); returns (R, P, F, dKE, extra)."""
    P = P + 0.5 * dt * F
    R, P = free_ring_step(R, P, m, C, w, dt / 2, box3)
    P, dKE = pile_l_step(P, m, C, gamma, dt, kT, noise)
    R, P = free_ring_step(R, P, m, C, w, dt / 2, box3)
    F, extra = force_fn(R)
    P = P + 0.5 * dt * F
    return R, P, F, dKE, extra


def min_image_unwrap(prev, cur, box3):
    return prev + np.remainder(cur - prev + box3 / 2, box3) - box3 / 2


def centroid_drift(R, P, m, box3, va, h):
    """Parrinello-Rahman drift of the centroid mode only (pimd.py:385-398):
    every bead moves by dR_c = R_c (e^x - 1) + h v_c e^(x/2) sinh(x/2)/(x/2),
    x = va h, with R_c the centroid of the beads unwrapped onto bead 0."""
    x = va * h
    Rc = unwrap_across_beads(R, box3).mean(0)
    vc = (P / m).mean(0)
    dRc = Rc * np.expm1(x) + h * vc * np.exp(x / 2) * sinhx_x(x / 2)
    return R + dRc[None]


def internal_ring_step(R, P, m, C, w, h, box3):
    """Exact free propagation of the non-centroid ring-polymer modes only
    (pimd.py:400-415); the centroid normal mode is left as it is."""
    R = unwrap_across_beads(R, box3)
    Q = np.tensordot(C.T, R, axes=(1, 0))
    Pn = np.tensordot(C.T, P, axes=(1, 0))
    w = w[:, None, None]
    c, s = np.cos(w * h), np.sin(w * h)
    sw = np.where(w == 0, 1.0, w)
    Qn, Pm = Q.copy(), Pn.copy()
    Qn[1:] = Q[1:] * c[1:] + Pn[1:] * s[1:] / (m * sw[1:])
    Pm[1:] = Pn[1:] * c[1:] - m * sw[1:] * Q[1:] * s[1:]
    return np.tensordot(C, Qn, axes=(1, 0)), np.tensordot(C, Pm, axes=(1, 0))


class NPTPIMDState:
    """NPT-PIMD state (pimd.py:253-296, init_fn 417-441): beads R, P, F
    (P, N, 3); log box scales Rb, momenta Pb, masses Mb = n_g (N + 1) kT
    tau_p^2 per coupled group; the cached centroid-virial dU/d(eps) per group;
    thermostat and box-thermostat work.  force_fn(R, box) -> (F, W_beads)
    with W_beads (P, 3, 3) the per-bead virials W = -sum r (x) f of the
    per-bead energies (their sum is n_bead times the bead-averaged energy)."""

    def __init__(self, R, P, F, W_beads, m, box, pressure, kT, tau_p, gid):
        self.R, self.P, self.F, self.m = R.copy(), P.copy(), F.copy(), m
        self.ref = np.asarray(box, float).copy()
        self.gid = np.asarray(gid)
        self.G = int(self.gid.max()) + 1
        self.ngrp = np.array([(self.gid == g).sum() for g in range(self.G)], float)
        N = R.shape[1]
        self.Rb = np.zeros(self.G)
        self.Pb = np.zeros(self.G)
        self.Mb = self.ngrp * (N + 1) * kT * tau_p ** 2
        self.pressure = pressure
        self.twork = 0.0
        self.btwork = 0.0
        self.dUde = self.centroid_dU_deps(R, F, W_beads, self.box())

    def box(self):
        return self.ref * np.array([np.exp(self.Rb[g]) if g >= 0 else 1.0 for g in self.gid])

    def axis_rate(self):
        vb = self.Pb / self.Mb
        return np.array([vb[g] if g >= 0 else 0.0 for g in self.gid]), float((self.ngrp * vb).sum())

    def centroid_dU_deps(self, R, F, W_beads, box3):
        """(dU/d eps_g + the internal-mode virial) / n_bead (pimd.py:332-350)."""
        nb = R.shape[0]
        Ruw = unwrap_across_beads(R, box3)
        internal = ((Ruw - Ruw.mean(0)) * F).sum((0, 1))
        out = np.zeros(self.G)
        for a in range(3):
            if self.gid[a] >= 0:
                out[self.gid[a]] += -W_beads[:, a, a].sum() + internal[a]
        return out / nb

    def box_force(self, V, Nf):
        """Box-momentum driver from the centroid momenta (pimd.py:366-373)."""
        KE2 = (self.P.mean(0) ** 2 / self.m).sum(0)
        tot = KE2.sum()
        grp = np.array([KE2[self.gid == g].sum() for g in range(self.G)])
        return grp + (self.ngrp / Nf) * tot - self.dUde - self.pressure * V * self.ngrp


def npt_pimd_step(st: NPTPIMDState, dt, kT, C, w, gamma, gamma_box, noise, noise_box, force_fn):
    """One step_fn of npt_langevin_pimd (pimd.py:443-516); noise (P, N, 3)
    and noise_box (G,) ~ N(0, 1).  Returns the per-bead virials."""
    N = st.R.shape[1]
    Nf = 3.0 * N
    h = dt / 2

    def kick(P, F):  # exp_iL2_pimd (pimd.py:375-383)
        va, tr = st.axis_rate()
        x = (va + tr / Nf) * h
        Pc, Fc = P.mean(0), F.mean(0)
        Pc_new = Pc * np.exp(-x) + h * Fc * sinhx_x(x / 2) * np.exp(-x / 2)
        return Pc_new[None] + (P - Pc[None]) + h * (F - Fc[None])

    st.Pb = st.Pb + h * st.box_force(np.prod(st.box()), Nf)
    st.P = kick(st.P, st.F)
    st.Rb = st.Rb + h * st.Pb / st.Mb
    box = st.box()
    st.R = centroid_drift(st.R, st.P, st.m, box, st.axis_rate()[0], h)
    st.R, st.P = internal_ring_step(st.R, st.P, st.m, C, w, h, box)
    st.P, dke = pile_l_step(st.P, st.m, C, gamma, dt, kT, noise)
    st.twork += dke
    c1 = np.exp(-gamma_box * dt)
    c2 = np.sqrt(max(kT * (1.0 - c1 ** 2), 0.0))
    Pb_old = st.Pb
    st.Pb = c1 * st.Pb + c2 * np.sqrt(st.Mb) * noise_box
    st.btwork += 0.5 * float(((st.Pb ** 2 - Pb_old ** 2) / st.Mb).sum())
    st.Rb = st.Rb + h * st.Pb / st.Mb
    box = st.box()
    st.R = centroid_drift(st.R, st.P, st.m, box, st.axis_rate()[0], h)
    st.R, st.P = internal_ring_step(st.R, st.P, st.m, C, w, h, box)
    st.F, W = force_fn(st.R, box)
    st.dUde = st.centroid_dU_deps(st.R, st.F, W, box)
    st.P = kick(st.P, st.F)
    st.Pb = st.Pb + h * st.box_force(np.prod(box), Nf)
    return W
