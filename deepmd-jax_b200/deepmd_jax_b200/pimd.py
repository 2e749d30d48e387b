"""Ring-polymer helpers of the reference's pimd module (deepmd_jax/pimd.py),
on the host in numpy: the normal-mode transform the engine is built with,
and the bead unwrapping, centroid and spring energy used to post-process a
PIMD trajectory (`Simulation.run` returns bead positions (steps, P, N, 3)).
The integrators themselves run on the device (dpb_md_*)."""
from __future__ import annotations

import numpy as np

HBAR = 6.582119569e-16 * 1e15  # eV fs (deepmd_jax/pimd.py:19)


def normal_mode_transform(n_bead, kT):
    """(freqs (P,), C (P, P)): ring-polymer normal-mode angular frequencies
    (fs^-1) and the orthogonal primitive <- normal-mode transform, from the
    eigenpairs of the ring's circulant matrix sorted by eigenvalue, the
    centroid eigenvalue set to zero (deepmd_jax/pimd.py:22-44)."""
    ring_poly_freq = n_bead * kT / HBAR
    A = 2 * np.eye(n_bead) - np.roll(np.eye(n_bead), 1, axis=0) - np.roll(np.eye(n_bead), -1, axis=0)
    eva, eve = np.linalg.eigh(A)
    order = np.argsort(eva)
    eva = eva[order]
    eve = eve[:, order]
    if n_bead >= 2:
        eva[0] = 0.0
    return ring_poly_freq * np.sqrt(np.maximum(eva, 0.0)), eve


def _minimg(delta, box):
    box = np.asarray(box, dtype=np.float64)
    if box.size == 3:
        b = box.reshape(3)
        return delta - b * np.round(delta / b)
    frac = delta @ np.linalg.inv(box)
    return (frac - np.round(frac)) @ box


def unwrap_across_beads(coord, box):
    """Every bead moved by whole box vectors onto bead 0's periodic image
    (deepmd_jax/pimd.py:210-227); coord (P, N, 3), box (3,) or (3, 3)."""
    coord = np.asarray(coord, dtype=np.float64)
    ref = coord[0:1]
    return ref + _minimg(coord - ref, box)


def centroid(coord, box):
    """Ring-polymer centroid (N, 3) with the beads unwrapped first
    (deepmd_jax/pimd.py:241-248)."""
    return unwrap_across_beads(coord, box).mean(axis=0)


def spring_energy(R, mass, box, omega_P):
    """0.5 m omega_P^2 sum over beads of (R_b - R_{b-1})^2 on the unwrapped
    ring (deepmd_jax/pimd.py:82-89); R (P, N, 3), mass (N, 1) in eV fs^2 /
    A^2, omega_P in fs^-1."""
    Ru = unwrap_across_beads(R, box)
    dR = Ru - np.roll(Ru, 1, axis=0)
    return 0.5 * omega_P ** 2 * float((np.asarray(mass) * dR ** 2).sum())


def unwrap_step_position(previous_position, current_position, box):
    """current_position on the periodic image nearest previous_position
    (deepmd_jax/pimd.py:228-238)."""
    prev = np.asarray(previous_position, dtype=np.float64)
    return prev + _minimg(np.asarray(current_position, dtype=np.float64) - prev, box)
