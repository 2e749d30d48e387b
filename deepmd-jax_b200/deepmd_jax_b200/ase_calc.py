"""ASE calculator with the reference's interface (deepmd_jax/ase_calc.py:18-144),
evaluated by libdpb200 on the GPU.

``DPJaxCalculator(model_path, type_idx)`` provides energy, forces and stress
of an ``ase.Atoms`` (any periodic cell; a general one is evaluated through
the open ghost-atom system of ``lattice.ghost_eval``, V = |det cell|).  The reference takes the stress as
jax_md.quantity.stress, -(1/V) dU/d(eps), and returns its negative in Voigt
order (xx, yy, zz, yz, xz, xy); with the virial W = -sum r (x) dE/dr that the
adjoint produces, dU/d(eps) = -W, so the returned stress is -W / V.

When ASE is installed the class derives from its Calculator; otherwise from a
small stand-in with the same get_potential_energy / get_forces / get_stress
entry points (ASE is not a dependency of this library).
"""
from __future__ import annotations

import numpy as np

from .dpmodel import DPModel, box_diagonal, general_box
from .utils import load_model

try:  # pragma: no cover - depends on the environment
    from ase.calculators.calculator import Calculator, all_changes
except ImportError:  # stand-in with the entry points callers use
    all_changes = ["positions", "numbers", "cell", "pbc"]

    class Calculator:
        implemented_properties: list = []

        def __init__(self, **kwargs):
            self.atoms = None
            self.results = {}

        def get_property(self, name, atoms=None):
            self.calculate(atoms)
            return self.results[name]

        def get_potential_energy(self, atoms=None, force_consistent=False):
            return self.get_property("energy", atoms)

        def get_forces(self, atoms=None):
            return self.get_property("forces", atoms)

        def get_stress(self, atoms=None):
            return self.get_property("stress", atoms)


class DPJaxCalculator(Calculator):
    implemented_properties = ["energy", "forces", "stress"]

    def __init__(self, model_path, type_idx=None, precision="fp32", **kwargs):
        super().__init__(**kwargs)
        self.atoms = None
        model, variables = load_model(model_path)
        self._params, self._variables = model.params, variables
        if self._params.get("type", "energy") != "energy":
            raise NotImplementedError("DPLR / atomic models are not implemented in the ASE calculator.")
        t = np.asarray(type_idx).astype(int)
        ct = self._params.get("chemical_types")
        if ct is not None:
            unknown = set(t.tolist()) - set(ct)
            if unknown:
                raise ValueError('Atomic numbers %s in type_idx are not in model.params["chemical_types"]=%s'
                                 % (sorted(unknown), ct))
            z2i = {z: i for i, z in enumerate(ct)}
            t = np.array([z2i[z] for z in t], dtype=int)
        self._type_idx = t
        self._model = DPModel(self._params, precision=precision)

    def calculate(self, atoms=None, properties=None, system_changes=all_changes):
        if atoms is not None:
            self.atoms = atoms.copy()
        cell = np.asarray(self.atoms.get_cell(complete=True), dtype=np.float64)
        box = box_diagonal(cell) if general_box(cell) is None else cell  # general cells: lattice.ghost_eval
        pos = np.asarray(self.atoms.get_positions(), dtype=np.float64)
        E, F, W = self._model.energy_force_virial(self._variables, pos, box, {"type_idx": tuple(self._type_idx)})
        V = abs(float(np.linalg.det(cell)))
        self.results["energy"] = float(E)
        self.results["forces"] = np.asarray(F)
        self.results["stress"] = -np.array([W[0, 0], W[1, 1], W[2, 2], W[1, 2], W[0, 2], W[0, 1]]) / V
