"""Golden vectors for embedding / fitting shapes other than the benchmark's,
from the UNMODIFIED reference model source on the torch-backed jax/flax
stand-in (same machinery as make_golden.py), written to golden_shapes.npz:

  F  embed (24, 48, 96), fit (200, 200, 200), axis 12   (dt on layers 1, 2)
  G  embed (16, 32, 64), fit (240, 120, 240), axis 16   (unequal fitting widths: no dt)
  H  embed (32, 16, 32, 64), fit (64, 64), axis 8       (four layers; 32 -> 16 is the
                                                          mean-pooled narrowing residual)
  I  F with a compressed-embedding table of width 96

every parameter non-trivial (randomize_model), on the 192-atom water box
(several periodic images per pair) and, for F, on a 1,536-atom box through a
neighbour list (key L).

Usage:  python tests/golden/make_golden_shapes.py /path/to/deepmd-jax   (the source checkout)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import (compressed_variant, randomize_model, ref_energy_force,  # noqa: E402
                         typed_to_nbrs_nm)
from deepmd_jax_b200.systems import init_dp_params, nnbrs_rule, water_box  # noqa: E402
from oracle import nlist as onl  # noqa: E402

SHAPES = {
    "F": dict(embed_widths=(24, 48, 96), fit_widths=(200, 200, 200), axis=12),
    "G": dict(embed_widths=(16, 32, 64), fit_widths=(240, 120, 240), axis=16),
    "H": dict(embed_widths=(32, 16, 32, 64), fit_widths=(64, 64), axis=8),
}


def shape_models():
    """The models of golden_shapes.npz, rebuilt deterministically."""
    w = water_box(4, 12.42, seed=0)
    nn = nnbrs_rule(w["position"], w["box"], w["type_idx"], 6.0)
    out = {}
    for k, (name, kw) in enumerate(sorted(SHAPES.items())):
        out[name] = randomize_model(*init_dp_params(nnbrs=nn, seed=20 + k, **kw), seed=30 + k)
    out["I"] = compressed_variant(*out["F"], seed=40)
    return out


def main(ref_root):
    import jaxshim
    ref = jaxshim.load_reference(ref_root)
    models = shape_models()
    w = water_box(4, 12.42, seed=0)
    out = dict(pos=w["position"], box=w["box"], type=w["type_idx"])
    for name, (p, v) in models.items():
        E, F = ref_energy_force(ref, p, v, w["position"], w["box"], w["type_idx"])
        out[name + "_E"], out[name + "_F"] = E, F
        print(name, E)
    # F through a neighbour list on a 1,536-atom box
    sel = [46, 92]
    wL = water_box(8, 24.83, seed=7)
    cnt = np.bincount(wL["type_idx"], minlength=2)
    c = onl.canonicalize(wL["position"], wL["box"], wL["type_idx"])
    typed, _, ovf = onl.typed_nlist(c, wL["box"].astype(np.float32), onl.cutoff_sq(6.3), cnt, sel)
    assert not ovf
    p, v = models["F"]
    EL, FL = ref_energy_force(ref, p, v, wL["position"], wL["box"], wL["type_idx"],
                              nbrs_nm=typed_to_nbrs_nm(typed, cnt, sel))
    out.update(L_pos=wL["position"], L_box=wL["box"], L_type=wL["type_idx"], L_E=EL, L_F=FL, L_nbrs=typed)
    print("F list", EL)
    np.savez_compressed(os.path.join(HERE, "golden_shapes.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path to the deepmd-jax source checkout>" % os.path.basename(sys.argv[0]))
    main(sys.argv[1])
