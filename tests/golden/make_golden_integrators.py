"""Generate golden steps of the reference's own integrators.

Runs the UNMODIFIED reference integrator source — the NVT ring-polymer step
(deepmd_jax/pimd.py:114-207), the NPT ring-polymer step with the Langevin
barostat (pimd.py:299-518), the classical BAOAB Langevin step with fixed
atoms (deepmd_jax/routine.py:46-107), the MTK NPT step with coupled axes
(routine.py:230-426) and the fixed-atom wrapper of NVE and Nose-Hoover NVT
(routine.py:110-158) — in float64 on the torch-backed jax stand-in of
jaxshim.py, and writes golden_integrators.npz next to this file.

The potential is a smooth Gaussian pair repulsion under the minimum image,
evaluated per bead and averaged over beads as the reference's energy_fn is
(md.py:416-444), with the strain handled through the `perturbation` argument
(coordinates and box scaled together, md.py:431-434).  The Gaussian noise the
steps draw is fixed in advance (seeded numpy) and saved, so the oracle can
replay the same step.  What the reference takes from jax_md (absent here, a
third-party dependency) is restated from its published definitions:
momentum_step p += dt F, position_step r = shift(r, dt p / m),
canonicalize_force = -grad of an energy, canonicalize_mass = identity for an
(N, 1) mass, the volume and kinetic energy of `quantity`; the Nose-Hoover
chain the NPT step calls (jax_md's nose_hoover_chain, with one chain step
and one Suzuki-Yoshida step) is the oracle's own restatement (oracle/
integrators.py NHChain), so the NPT fixture pins the barostat, the coupled
axes and the step order of routine.py but not the chain substep itself;
likewise jax_md's nve / nvt_nose_hoover (velocity Verlet, chain half steps
around it) are restated, so the fixed-atom fixtures pin the wrapper's
masking and its chain degrees of freedom, mass and kinetic energy.
jax.grad / jax.value_and_grad are torch autograd.

Usage:  python tests/golden/make_golden_integrators.py /path/to/deepmd-jax   (the source checkout)
"""
from __future__ import annotations

import dataclasses
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import jaxshim  # noqa: E402
from jaxshim import J, JArray  # noqa: E402

PAIR_A, PAIR_S2 = 0.8, 2.0   # phi(r) = A exp(-r^2 / s2), eV and A^2


def pair_energy(R, box, perturbation=1.0):
    """Bead-averaged Gaussian pair energy of R (P, N, 3) in an orthorhombic
    box (3,), coordinates and box scaled by `perturbation`; torch float64."""
    R = torch.as_tensor(R)
    L = torch.as_tensor(box) * perturbation
    X = R * perturbation
    d = X[:, :, None, :] - X[:, None, :, :]
    d = d - L * torch.round(d / L)
    r2 = (d * d).sum(-1)
    n = R.shape[1]
    off = ~torch.eye(n, dtype=torch.bool)
    e = 0.5 * (PAIR_A * torch.exp(-r2 / PAIR_S2))[:, off].sum()
    return e / R.shape[0]


class _SizeInt(int):
    """numpy's `.size` (element count) that is still callable like torch's
    `.size()`, for the reference's `box.size == 3` tests."""

    def __new__(cls, t):
        obj = int.__new__(cls, t.numel())
        obj._shape = t.shape
        return obj

    def __call__(self, dim=None):
        return self._shape if dim is None else self._shape[dim]


class _F64:
    """jnp.float32 of the stand-in: a dtype, and callable as a constructor."""

    def __call__(self, x):
        return J(x, torch.float64)


def _install_extras():
    jaxshim.install()
    jnp, jax = jaxshim.jnp, jaxshim.jax
    f64 = _F64()
    base_dtype = jaxshim._dtype
    jaxshim._dtype = lambda dt: torch.float64 if isinstance(dt, _F64) else base_dtype(dt)
    jnp.float32 = f64
    jnp.isscalar = lambda x: np.isscalar(x)
    JArray.size = property(lambda self: _SizeInt(self))
    JArray.at = property(lambda self: _At(self))
    JArray.mean = lambda self, axis=None, keepdims=False: (
        torch.Tensor.mean(self) if axis is None else torch.Tensor.mean(self, dim=axis, keepdim=keepdims))
    jaxshim.jrandom.split = lambda key, n=2: tuple([key] * n)

    def tensordot(a, b, axes):  # numpy's axes=(i, j) pairs single axes
        if isinstance(axes, (tuple, list)) and len(axes) == 2 and all(isinstance(x, int) for x in axes):
            axes = ([axes[0]], [axes[1]])
        return torch.tensordot(*jaxshim._promote(J(a), J(b)), dims=axes).as_subclass(JArray)
    jnp.tensordot = tensordot

    def grad(f, argnums=0):
        def g(*args, **kw):
            return value_and_grad(f, argnums)(*args, **kw)[1]
        return g

    def value_and_grad(f, argnums=0):
        nums = (argnums,) if isinstance(argnums, int) else tuple(argnums)

        def g(*args, **kw):
            args = list(args)
            xs = []
            for i in nums:
                x = torch.as_tensor(args[i], dtype=torch.float64).detach().clone().requires_grad_(True)
                args[i] = x.as_subclass(JArray)
                xs.append(x)
            y = f(*args, **kw)
            gs = torch.autograd.grad(y, xs)
            gs = tuple(t.detach().as_subclass(JArray) for t in gs)
            return y.detach(), (gs[0] if isinstance(argnums, int) else gs)
        return g

    jax.grad = grad
    jax.value_and_grad = value_and_grad

    simulate = types.SimpleNamespace(
        NVTNoseHooverState=object, NoseHooverChain=object,
        momentum_step=lambda st, dt: st.set(momentum=st.momentum + dt * st.force),
        position_step=lambda st, shift_fn, dt, **kw: st.set(
            position=shift_fn(st.position, dt * st.momentum / st.mass, **kw)),
        canonicalize_mass=lambda st: st,
        initialize_momenta=lambda st, key, kT: st.set(momentum=_centred(
            torch.sqrt(torch.as_tensor(st.mass) * kT) * jaxshim.jrandom.normal(key, tuple(st.position.shape)))),
        kinetic_energy=_kinetic,
        nve=_nve,
        nvt_nose_hoover=_nvt_nose_hoover,
        default_nhc_kwargs=lambda tau, kw: {"chain_length": 3, "chain_steps": 2, "sy_steps": 3, "tau": tau,
                                            **(kw or {})},
        nose_hoover_chain=_nose_hoover_chain,
    )
    quantity = types.SimpleNamespace(
        canonicalize_force=lambda fn: (lambda R, **kw: -grad(fn)(R, **kw)),
        volume=lambda dim, box: torch.prod(torch.as_tensor(box)).as_subclass(JArray),
        kinetic_energy=lambda momentum=None, mass=None: (0.5 * (torch.as_tensor(momentum) ** 2
                                                                / torch.as_tensor(mass)).sum()).as_subclass(JArray),
        count_dof=lambda R: int(np.prod(tuple(torch.as_tensor(R).shape))))
    util = types.SimpleNamespace(high_precision_sum=lambda x, axis=None: torch.sum(torch.as_tensor(x), dim=axis)
                                 .as_subclass(JArray))
    jax_md = sys.modules["jax_md"]
    jax_md.simulate = simulate
    jax_md.quantity = quantity
    jax_md.util = util
    sys.modules["jax_md.simulate"] = simulate


def _centred(p):
    p = torch.as_tensor(p)
    return (p - torch.mean(p, dim=0, keepdim=True)).as_subclass(JArray)


def _noise_queue(arrays):
    q = list(arrays)

    def fn(shape):
        a = q.pop(0)
        assert tuple(a.shape) == tuple(shape), (a.shape, shape)
        return torch.as_tensor(a)
    return fn


def _with_set(cls):
    cls.set = lambda self, **kw: dataclasses.replace(self, **kw)


@dataclasses.dataclass
class _Chain:
    """jax_md's NoseHooverChain state: xi, p, Q, tau, KE, DOF."""
    position: object
    momentum: object
    mass: object
    tau: float
    kinetic_energy: object
    degrees_of_freedom: float

    def set(self, **kw):
        return dataclasses.replace(self, **kw)


@dataclasses.dataclass
class _NVEState:
    position: object
    momentum: object
    force: object
    mass: object

    velocity = property(lambda self: self.momentum / self.mass)

    def set(self, **kw):
        return dataclasses.replace(self, **kw)


@dataclasses.dataclass
class _NVTState(_NVEState):
    chain: object = None


def _kinetic(st):
    return (0.5 * (torch.as_tensor(st.momentum) ** 2 / torch.as_tensor(st.mass)).sum()).as_subclass(JArray)


def _momenta(R, mass, kT):
    """jax_md initialize_momenta: sqrt(m kT) N(0, 1), mean momentum removed."""
    p = torch.sqrt(torch.as_tensor(mass) * kT) * jaxshim.jrandom.normal(0, tuple(torch.as_tensor(R).shape))
    return _centred(p)


def _velocity_verlet(force_fn, shift_fn, dt, st, **kw):
    st = st.set(momentum=st.momentum + 0.5 * dt * st.force)
    st = st.set(position=shift_fn(st.position, dt * st.momentum / st.mass, **kw))
    st = st.set(force=force_fn(st.position, **kw))
    return st.set(momentum=st.momentum + 0.5 * dt * st.force)


def _nve(energy_fn, shift_fn, dt, **kw):
    """jax_md.simulate.nve: velocity Verlet."""
    force_fn = lambda R, **k: -jaxshim.jax.grad(energy_fn)(R, **k)  # noqa: E731

    def init_fn(key, R, mass=1.0, kT=0.0, **k):
        return _NVEState(R, _momenta(R, mass, kT), force_fn(R, **k), mass)

    def apply_fn(st, **k):
        return _velocity_verlet(force_fn, shift_fn, dt, st, **k)
    return init_fn, apply_fn


def _nvt_nose_hoover(energy_fn, shift_fn, dt, kT, tau=None, chain_length=3, chain_steps=1, sy_steps=1):
    """jax_md.simulate.nvt_nose_hoover: chain half step, velocity Verlet,
    chain half step, the chain masses refreshed first."""
    force_fn = lambda R, **k: -jaxshim.jax.grad(energy_fn)(R, **k)  # noqa: E731
    chain = _nose_hoover_chain(dt, chain_length, chain_steps, sy_steps, tau)

    def init_fn(key, R, mass=1.0, **k):
        st = _NVTState(R, _momenta(R, mass, kT), force_fn(R, **k), mass)
        c = chain.initialize(int(np.prod(tuple(torch.as_tensor(R).shape))), float(_kinetic(st)), kT)
        return st.set(chain=c.set(mass=J(c.mass)))

    def apply_fn(st, **k):
        c = chain.update_mass(st.chain, kT)
        p, c = chain.half_step(st.momentum, c, kT)
        st = _velocity_verlet(force_fn, shift_fn, dt, st.set(momentum=p), **k)
        c = c.set(kinetic_energy=float(_kinetic(st)))
        p, c = chain.half_step(st.momentum, c, kT)
        return st.set(momentum=p, chain=c)
    return init_fn, apply_fn


class _At:
    """x.at[i].multiply(v) / .set(v) / .add(v) of jax arrays, out of place."""

    def __init__(self, x):
        self.x = x

    def __getitem__(self, idx):
        x = self.x

        def upd(fn):
            y = torch.as_tensor(x).clone()
            y[idx] = fn(y[idx])
            return y.as_subclass(JArray)
        return types.SimpleNamespace(multiply=lambda v: upd(lambda a: a * v), set=lambda v: upd(lambda a: a * 0 + v),
                                     add=lambda v: upd(lambda a: a + v))


def _nose_hoover_chain(dt, chain_length=3, chain_steps=1, sy_steps=1, tau=100.0):
    """initialize / update_mass / half_step of jax_md.simulate.nose_hoover_chain
    for chain_steps = sy_steps = 1, the substep taken from the oracle."""
    from oracle.integrators import NHChain
    assert chain_steps == 1 and sy_steps == 1
    L, dt, tau = chain_length, float(dt), float(tau)

    def masses(kT, dof):
        Q = kT * tau ** 2 * np.ones(L)
        Q[0] *= dof
        return Q

    def initialize(dof, KE, kT):
        return _Chain(np.zeros(L), np.zeros(L), masses(kT, dof), tau, float(KE), float(dof))

    def update_mass(c, kT):
        return c.set(mass=masses(kT, c.degrees_of_freedom))

    def half_step(P, c, kT):
        ch = NHChain(L, c.degrees_of_freedom, kT, tau, float(c.kinetic_energy))
        ch.xi, ch.p, ch.Q = np.array(c.position), np.array(c.momentum), np.array(c.mass)
        Pn = ch.substep(dt, np.asarray(torch.as_tensor(P)), kT)
        return J(Pn), c.set(position=ch.xi, momentum=ch.p, kinetic_energy=ch.KE)
    return types.SimpleNamespace(initialize=initialize, update_mass=update_mass, half_step=half_step)


def main(ref_root):
    import importlib
    _install_extras()
    pkg = types.ModuleType("deepmd_jax")
    pkg.__path__ = [str(ref_root) + "/deepmd_jax"]
    sys.modules["deepmd_jax"] = pkg
    pimd = importlib.import_module("deepmd_jax.pimd")
    routine = importlib.import_module("deepmd_jax.routine")
    for c in (pimd.PIMDLangevinState, pimd.PIMDNPTLangevinState, routine.NVTLangevinStateWithWork,
              routine.CachedNPTNoseHooverState):
        _with_set(c)

    rng = np.random.default_rng(2024)
    P, N = 4, 12
    box = np.array([6.3, 7.1, 6.7])
    kT = 300.0 * 8.617333e-5
    mass = rng.uniform(1.0, 16.0, size=(N, 1)) * 103.6427
    centres = rng.uniform(0, 1, size=(N, 3)) * box
    R0 = centres[None] + rng.normal(scale=0.05, size=(P, N, 3))
    P0 = np.sqrt(mass * kT * P) * rng.normal(size=(P, N, 3))
    freqs, C = pimd.normal_mode_transform(P, kT)
    freqs, C = np.asarray(freqs, dtype=np.float64), np.asarray(C, dtype=np.float64)
    gamma = 2.0 * freqs
    gamma[0] = 1.0 / 100.0
    dt = 0.5

    def energy_fn(R, box=None, perturbation=1.0, **kw):
        return pair_energy(R, box, perturbation).as_subclass(JArray)

    out = dict(P=P, N=N, box=box, kT=kT, mass=mass, R0=R0, P0=P0, C=C, freqs=freqs, gamma=gamma, dt=dt,
               pair=np.array([PAIR_A, PAIR_S2]))

    # --- NVT ring-polymer BAOAB step (pimd.py:193-205)
    init_fn, step_fn = pimd.nvt_langevin_pimd(energy_fn, None, dt, kT, J(box), J(gamma), J(C), J(freqs))
    F0 = -jaxshim.jax.grad(lambda R: P * energy_fn(R, box=J(box)))(J(R0))
    st = pimd.PIMDLangevinState(position=J(R0), momentum=J(P0), force=F0, mass=J(mass), rng=0,
                                thermostat_work=J(0.0))
    noise = rng.normal(size=(P, N, 3))
    jaxshim._NOISE["fn"] = _noise_queue([noise])
    st = step_fn(st)
    out.update(nvt_noise=noise, nvt_R=st.position.numpy(), nvt_P=st.momentum.numpy(), nvt_F=st.force.numpy(),
               nvt_work=float(st.thermostat_work))

    # --- NPT ring-polymer step, Langevin barostat (pimd.py:443-516), axes x,y coupled and z alone
    gid = np.array([0, 0, 1])
    G = 2
    membership = np.zeros((3, G))
    membership[[0, 1, 2], gid] = 1.0
    n_per_group = membership.sum(0)
    pressure, tau_p = 50.0 * 6.241509e-7, 200.0
    init_fn, step_fn = pimd.npt_langevin_pimd(
        energy_fn, lambda R, dR, **kw: R + dR, dt, pressure=pressure, kT=kT, gamma_P=J(gamma),
        gamma_box=1.0 / tau_p, nm_trans=J(C), nm_freqs=J(freqs), membership=J(membership),
        n_per_group=J(n_per_group), group_ids=J(gid), tau_p=tau_p)
    jaxshim._NOISE["fn"] = _noise_queue([np.zeros((P, N, 3))])    # momenta of init_fn, replaced below
    st = init_fn(0, J(R0), J(box), mass=J(mass))
    st = st.set(momentum=J(P0), box_momentum=J(np.array([0.3, -0.2])))
    noise, noise_b = rng.normal(size=(P, N, 3)), rng.normal(size=(G,))
    out.update(npt_gid=gid, npt_pressure=pressure, npt_tau_p=tau_p, npt_Pb0=np.array([0.3, -0.2]),
               npt_dUdV0=st.dUdV.numpy(), npt_Mb=st.box_mass.numpy())
    jaxshim._NOISE["fn"] = _noise_queue([noise, noise_b])
    st = step_fn(st)
    out.update(npt_noise=noise, npt_noise_b=noise_b, npt_R=st.position.numpy(), npt_P=st.momentum.numpy(),
               npt_F=st.force.numpy(), npt_Rb=st.box_position.numpy(), npt_Pb=st.box_momentum.numpy(),
               npt_dUdV=st.dUdV.numpy(), npt_work=float(st.thermostat_work),
               npt_box_work=float(st.box_thermostat_work))

    # --- classical BAOAB Langevin with fixed atoms (routine.py:46-107), bead 0 as the system
    mobile = np.ones(N, dtype=bool)
    mobile[[1, 5]] = False
    mob = J(mobile.astype(np.float64))[:, None]

    def e1(R, **kw):  # one replica; fixed atoms' coordinates under stop_gradient (md.py:428-430)
        R = torch.where(mob.bool(), R, R.detach())
        return pair_energy(R[None], J(box)).as_subclass(JArray)

    def shift(R, dR, **kw):  # md.py:231-234: fixed atoms keep their position
        return torch.where(mob.bool(), R + dR, R).as_subclass(JArray)

    init_fn, step_fn = routine.nvt_langevin(e1, shift, dt, kT, gamma=1.0 / 50.0, mobile_mask=mobile)
    r0, p0 = R0[0], P0[0] / np.sqrt(P) * mobile[:, None]
    f0 = -jaxshim.jax.grad(e1)(J(r0))
    st = routine.NVTLangevinStateWithWork(position=J(r0), momentum=J(p0), force=f0, mass=J(mass), rng=0,
                                          thermostat_work=J(0.0))
    noise = rng.normal(size=(N, 3))
    jaxshim._NOISE["fn"] = _noise_queue([noise])
    st = step_fn(st)
    out.update(lan_mobile=mobile, lan_r0=r0, lan_p0=p0, lan_noise=noise, lan_R=st.position.numpy(),
               lan_P=st.momentum.numpy(), lan_F=st.force.numpy(), lan_work=float(st.thermostat_work))

    # --- fixed atoms under NVE and Nose-Hoover NVT (routine.py:110-158), three steps each
    for name, make in (("fnve", lambda: routine.nve(e1, shift, dt, mobile_mask=J(mobile))),
                       ("fnvt", lambda: routine.nvt_nose_hoover(e1, shift, dt, kT, tau=60.0, chain_length=3,
                                                                chain_steps=1, sy_steps=1,
                                                                mobile_mask=J(mobile)))):
        init_fn, apply_fn = make()
        noise = rng.normal(size=(N, 3))
        jaxshim._NOISE["fn"] = _noise_queue([noise])
        st = init_fn(0, J(r0), mass=J(mass), kT=kT) if name == "fnve" else init_fn(0, J(r0), mass=J(mass))
        out[name + "_p0"] = st.momentum.numpy().copy()
        if name == "fnvt":
            out[name + "_Q0"] = np.asarray(st.chain.mass)
            out[name + "_KE0"] = float(st.chain.kinetic_energy)
        for _ in range(3):
            st = apply_fn(st)
        out[name + "_R"], out[name + "_P"] = st.position.numpy(), st.momentum.numpy()
        if name == "fnvt":
            out[name + "_xi"], out[name + "_pxi"] = np.asarray(st.chain.position), np.asarray(st.chain.momentum)

    # --- MTK NPT with NHC thermostat and barostat (routine.py:230-426), axes x alone, y,z coupled
    gid = np.array([0, 1, 1])
    tau_t, tau_p, pressure = 40.0, 150.0, 200.0 * 6.241509e-7
    init_fn, apply_fn = routine.npt_nose_hoover(
        lambda R, box=None, perturbation=1.0, **kw: energy_fn(R[None], box=box, perturbation=perturbation),
        lambda R, dR, **kw: R + dR, dt, pressure, kT,
        barostat_kwargs={"chain_length": 3, "chain_steps": 1, "sy_steps": 1, "tau": tau_p},
        thermostat_kwargs={"chain_length": 3, "chain_steps": 1, "sy_steps": 1, "tau": tau_t},
        couple_axes=((0,), (1, 2)))
    jaxshim._NOISE["fn"] = _noise_queue([np.zeros((N, 3))])      # momenta of init_fn, replaced below
    r0, p0 = R0[0], P0[0] / np.sqrt(P)
    st = init_fn(0, J(r0), J(box), mass=J(mass))
    st = st.set(momentum=J(p0), box_momentum=J(np.array([0.4, -0.3])),
                thermostat=st.thermostat.set(kinetic_energy=0.5 * float((p0 ** 2 / mass).sum())))
    out.update(mtk_gid=gid, mtk_tau_t=tau_t, mtk_tau_p=tau_p, mtk_pressure=pressure, mtk_Pb0=np.array([0.4, -0.3]),
               mtk_dUdV0=st.dUdV.numpy())
    for _ in range(3):
        st = apply_fn(st)
    out.update(mtk_R=st.position.numpy(), mtk_P=st.momentum.numpy(), mtk_F=st.force.numpy(),
               mtk_Rb=st.box_position.numpy(), mtk_Pb=st.box_momentum.numpy(), mtk_dUdV=st.dUdV.numpy(),
               mtk_xi=np.asarray(st.thermostat.position), mtk_pxi=np.asarray(st.thermostat.momentum),
               mtk_bxi=np.asarray(st.barostat.position), mtk_bpxi=np.asarray(st.barostat.momentum))

    np.savez_compressed(os.path.join(HERE, "golden_integrators.npz"), **out)
    print("nvt work", out["nvt_work"], "npt box", out["npt_Rb"], "lan work", out["lan_work"])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path to the deepmd-jax source checkout>" % os.path.basename(sys.argv[0]))
    main(sys.argv[1])
