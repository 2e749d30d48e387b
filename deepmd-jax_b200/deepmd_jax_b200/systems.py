"""Synthetic water systems and random-init se_a energy models.

These builders produce the inputs the benchmarks and tests run on: liquid-water
boxes (O on a jittered simple-cubic lattice, each H at the gas-phase geometry
with a random orientation) and a randomly initialised Deep Potential energy
model laid out exactly like the reference's ``model.pkl`` payload
(``DPModel.params`` plus ``variables['params']``; deepmd_jax/train.py:288-304,
deepmd_jax/dpmodel.py:50-81, deepmd_jax/utils.py:100-166).
"""
from __future__ import annotations

import numpy as np

MASS_O = 15.9994
MASS_H = 1.0078
MASS_UNIT_CONVERSION = 1.036427e2   # Dalton -> eV fs^2 / A^2 (deepmd_jax/md.py:24)
TEMP_UNIT_CONVERSION = 8.617333e-5  # Kelvin -> eV (deepmd_jax/md.py:25)
PRESS_UNIT_CONVERSION = 6.241509e-7  # bar -> eV / A^3 (deepmd_jax/md.py:26)
OH_BOND = 0.9572
HOH_ANGLE_DEG = 104.52


def _random_rotations(rng, n):
    """Uniform random rotation matrices from normalised Gaussian quaternions."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_box(n_side: int, box: float, seed: int = 0, n_water: int | None = None,
              temperature: float = 300.0, jitter: float = 0.1):
    """Liquid-water-like box.

    O atoms sit on the first ``n_water`` sites of an ``n_side``^3 simple-cubic
    lattice of spacing ``box / n_side`` with N(0, jitter) displacements; each
    molecule is written as (O, H, H) in that order, so the user atom order
    interleaves the two types.  Velocities are Maxwell-Boltzmann at
    ``temperature`` with the centre-of-mass motion removed.

    Returns dict(position (N,3) f64, velocity (N,3) f64, type_idx (N,) int,
    box (3,) f64, mass_per_type (2,), mass (N,)).
    """
    rng = np.random.default_rng(seed)
    if n_water is None:
        n_water = n_side ** 3
    a = box / n_side
    g = np.arange(n_side)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:n_water]
    O = (sites + 0.5) * a + rng.normal(scale=jitter, size=(n_water, 3))
    half = np.deg2rad(HOH_ANGLE_DEG) / 2
    local = OH_BOND * np.array([[np.sin(half), 0.0, np.cos(half)],
                                [-np.sin(half), 0.0, np.cos(half)]])
    Rm = _random_rotations(rng, n_water)
    H = O[:, None, :] + np.einsum("nij,hj->nhi", Rm, local)
    pos = np.concatenate([O[:, None, :], H], axis=1).reshape(-1, 3)
    type_idx = np.tile(np.array([0, 1, 1]), n_water)
    mass_per_type = np.array([MASS_O, MASS_H])
    mass = mass_per_type[type_idx]
    kT = temperature * TEMP_UNIT_CONVERSION
    m_int = mass * MASS_UNIT_CONVERSION
    vel = rng.normal(size=pos.shape) * np.sqrt(kT / m_int)[:, None]
    vel -= (vel * m_int[:, None]).sum(0) / m_int.sum()
    return dict(position=pos, velocity=vel, type_idx=type_idx,
                box=np.full(3, float(box)), mass_per_type=mass_per_type, mass=mass)


# Benchmark/test systems: (waters per side, box length in Angstrom).
WATER_CONFIGS = {
    "water192": (4, 12.42),
    "water12k": (16, 49.66),
    "water98k": (32, 99.3),
    "water1536": (8, 24.83),
}


def serving_water(n_water: int, seed: int = 0):
    """Water frame for the serving stream: first n_water sites of a
    ceil(n_water^(1/3))^3 lattice, box = 12.42 * (n_water / 64)^(1/3)."""
    n_side = int(np.ceil(n_water ** (1.0 / 3.0) - 1e-9))
    L = 12.42 * (n_water / 64.0) ** (1.0 / 3.0)
    return water_box(n_side, L, seed=seed, n_water=n_water)


def init_dp_params(ntypes: int = 2, embed_widths=(25, 50, 100), fit_widths=(240, 240, 240),
                   axis: int = 16, rcut: float = 6.0, nnbrs: float = 100.0, seed: int = 0,
                   sr_mean=None, sr_std=None, ebias=None, dtype=np.float32):
    """Random-init se_a energy model in the reference's parameter layout.

    Kernels are Xavier-normal (std = sqrt(2 / (fan_in + fan_out))), biases are
    zero, the fitting-net time-step vectors ``dt{k}`` follow the reference
    initialiser 0.1 + N(0, 0.001) (deepmd_jax/utils.py:93), ``Tbias`` is zero.
    Returns (params, variables) with ``variables = {'params': {...}}``.
    """
    rng = np.random.default_rng(seed)
    params = {
        "type": "energy",
        "atomic_data_prefix": None,
        "embed_widths": list(embed_widths),
        "embedMP_widths": None,
        "fit_widths": list(fit_widths),
        "axis": int(axis),
        "Ebias": np.zeros(ntypes, dtype) if ebias is None else np.asarray(ebias, dtype),
        "rcut": float(rcut),
        "use_2nd": True,
        "use_mp": False,
        "atomic": False,
        "hybrid": False,
        "nsel": None,
        "out_norm": 1.0,
        "ntypes": ntypes,
        "valid_types": np.arange(ntypes),
        "sr_mean": np.zeros(ntypes) if sr_mean is None else np.asarray(sr_mean, float),
        "sr_std": np.ones(ntypes) if sr_std is None else np.asarray(sr_std, float),
        "Nnbrs": float(nnbrs),
    }

    def dense(fan_in, fan_out):
        std = np.sqrt(2.0 / (fan_in + fan_out))
        return {"kernel": (rng.normal(size=(fan_in, fan_out)) * std).astype(dtype),
                "bias": np.zeros(fan_out, dtype)}

    var = {}
    for k in range(ntypes * ntypes):
        net, prev = {}, 1
        for li, w in enumerate(embed_widths):
            net["Dense_%d" % li] = dense(prev, w)
            prev = w
        var["embedding_net_%d" % k] = net
    W = embed_widths[-1]
    var["Tbias"] = np.zeros(W, dtype)
    for t in range(ntypes):
        net, prev = {}, axis * W
        for li, w in enumerate(fit_widths):
            net["Dense_%d" % li] = dense(prev, w)
            if li > 0 and fit_widths[li] == fit_widths[li - 1]:
                net["dt%d" % li] = (0.1 + rng.normal(scale=0.001, size=w)).astype(dtype)
            prev = w
        net["Dense_%d" % len(fit_widths)] = dense(prev, 1)
        var["fitting_net_%d" % t] = net
    return params, {"params": var}


def nnbrs_rule(position, box, type_idx, rcut):
    """Reference rule for params['Nnbrs'] (deepmd_jax/data.py:134): mean over
    atoms of the number of neighbours with s(r) > 0 (0 < r < rcut, all periodic
    images) plus one."""
    pos = np.asarray(position, float)
    L = np.asarray(box, float)
    n_img = int(np.ceil(rcut / L.min())) + 1
    rng_ = np.arange(-n_img, n_img + 1)
    shifts = np.stack(np.meshgrid(rng_, rng_, rng_, indexing="ij"), -1).reshape(-1, 3) * L
    d = pos[None, :, None, :] - pos[:, None, None, :] + shifts[None, None]
    r = np.linalg.norm(d, axis=-1)
    cnt = ((r > 1e-14) & (r < rcut)).sum(axis=(1, 2))
    return float(cnt.mean() + 1)
