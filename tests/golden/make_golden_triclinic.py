"""Golden vectors for general (triclinic) boxes, from the UNMODIFIED reference
model source on the torch-backed jax/flax stand-in (same machinery as
make_golden.py), written to golden_triclinic.npz.  The reference evaluates
such frames on its lattice path: displacements shifted into the
parallelepiped with ``shift(..., ortho=False)`` (deepmd_jax/utils.py:20-27)
and offset by the lattice candidates of ``compute_lattice_candidate``
(deepmd_jax/data.py:347-364).

  S  192-atom water, the 12.42 A cube's fractional coordinates in a sheared
     cell (every face wider than 2 rcut along its normal: one image per pair)
  U  96-atom water in a sheared cell narrower than 2 rcut (several images)

both with model B of make_golden.py (every parameter non-trivial).

Usage:  python tests/golden/make_golden_triclinic.py /path/to/deepmd-jax   (the source checkout)
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import golden_models  # noqa: E402
from deepmd_jax_b200.systems import water_box  # noqa: E402

CELLS = {
    # rows are the lattice vectors (coord = frac @ box, the reference's convention)
    "S": (dict(n=4, L=12.42, seed=0), np.array([[13.4, 0.0, 0.0], [3.1, 13.0, 0.0], [-2.2, 1.7, 13.2]])),
    "U": (dict(n=4, L=9.86, seed=5, n_water=32), np.array([[10.1, 0.0, 0.0], [2.6, 9.8, 0.0], [1.2, -2.1, 9.9]])),
}


def triclinic_frame(spec, B):
    """Water molecules of a cubic box carried into the cell B by their
    fractional coordinates."""
    kw = dict(spec)
    n, L, seed = kw.pop("n"), kw.pop("L"), kw.pop("seed")
    w = water_box(n, L, seed=seed, **kw)
    frac = w["position"] / L
    return frac @ B, w["type_idx"]


def ref_energy_force_box33(ref, params, variables, coord, box33, type_idx):
    dpmodel, data = ref["dpmodel"], ref["data"]
    from jaxshim import J
    model = dpmodel.DPModel(params)
    lattice = data.compute_lattice_candidate(J(np.asarray(box33, np.float64))[None], params["rcut"],
                                             print_info=False)
    static_args = {"type_idx": tuple(int(t) for t in type_idx), "use_neighbor_list": False, "lattice": lattice}
    c = J(np.asarray(coord, np.float64)).requires_grad_(True)
    E, _ = model.apply(variables, c, J(np.asarray(box33, np.float64)), static_args, None)
    g = torch.autograd.grad(E, c)[0]
    return float(E), (-g).detach().numpy().astype(np.float64)


def main(ref_root):
    import jaxshim
    ref = jaxshim.load_reference(ref_root)
    p, v = golden_models()["B"]
    out = {}
    for name, (spec, B) in CELLS.items():
        pos, types = triclinic_frame(spec, B)
        E, F = ref_energy_force_box33(ref, p, v, pos, B, types)
        out.update({name + "_pos": pos, name + "_box": B, name + "_type": types, name + "_E": E, name + "_F": F})
        print(name, len(types), E)
    np.savez_compressed(os.path.join(HERE, "golden_triclinic.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path to the deepmd-jax source checkout>" % os.path.basename(sys.argv[0]))
    main(sys.argv[1])
