"""Generate the golden vectors that pin the oracle to the reference.

Runs the UNMODIFIED reference model source (deepmd_jax/dpmodel.py,
deepmd_jax/utils.py, deepmd_jax/data.py:347-364 and deepmd_jax/pimd.py from a
reference checkout) in float64 on a torch-backed jax/flax stand-in
(jaxshim.py), with forces from torch autograd, and writes small .npz fixtures
next to this file.  jax itself is not installed in this environment; the
stand-in reproduces the jax semantics the model path relies on (see
jaxshim.py).  Neighbour lists fed to the reference model come from the
oracle's brute-force list (jax_md, which builds them in the reference, is a
third-party dependency that is absent).

Usage:  python tests/golden/make_golden.py /path/to/deepmd-jax   (the source checkout)
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "deepmd-jax_b200"))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from deepmd_jax_b200.systems import water_box, init_dp_params, nnbrs_rule  # noqa: E402
from oracle import nlist as onl  # noqa: E402
from oracle import philox  # noqa: E402


def randomize_model(params, variables, seed):
    """Give every parameter the reference model carries a non-trivial value
    (biases, Tbias, Ebias, per-type sr_mean/sr_std) so no term hides behind a
    zero."""
    rng = np.random.default_rng(seed)
    v = variables["params"]
    for name, net in v.items():
        if name == "Tbias":
            v[name] = (rng.normal(size=net.shape) * 0.1).astype(np.float32)
            continue
        for lname, layer in net.items():
            if isinstance(layer, dict) and "bias" in layer:
                layer["bias"] = (rng.normal(size=layer["bias"].shape) * 0.1).astype(np.float32)
    params["Ebias"] = rng.normal(size=params["ntypes"]).astype(np.float32)
    params["sr_mean"] = np.array([0.12, 0.07])
    params["sr_std"] = np.array([0.31, 0.22])
    return params, variables


def compressed_variant(params, variables, seed, ngrids=64):
    """Attach a random quintic table in the reference's compress_var layout
    (utils.py:269-286) so the compressed-embedding branch (utils.py:126-151)
    can be exercised without jax.jacfwd."""
    rng = np.random.default_rng(seed)
    params = dict(params)
    params["is_compressed"] = True
    W = params["embed_widths"][-1]
    cv = {}
    for k in range(params["ntypes"] ** 2):
        i = k // params["ntypes"]
        srmin = (0.0 - params["sr_mean"][i]) / params["sr_std"][i]
        srmax = (1.7 - params["sr_mean"][i]) / params["sr_std"][i]
        cv["embedding_net_%d" % k] = {
            "srmin": np.float32(srmin), "srmax": np.float32(srmax),
            "poly_coeff": (rng.normal(size=(ngrids, 6, W)) * 0.3).astype(np.float32)}
    variables = dict(variables)
    variables["compress_var"] = cv
    return params, variables


def hermite_compressed(params, variables, ngrids=256, rmin=0.5):
    """Attach compress_var tables built the way the reference's
    compress_model builds them (deepmd_jax/utils.py:250-297): on each of
    ``ngrids`` intervals of [srmin, srmax) = [(0 - mean)/std, (sr(rmin) -
    mean)/std) of the centre type, the quintic that matches the embedding
    net's value, first and second derivative at both ends (C2 piecewise
    quintic), stored as poly_coeff (ngrids, 6, W) in powers x0^(5-i).
    Values and derivatives come from the float64 oracle net and torch
    autograd."""
    import torch
    from oracle import model as om
    params = dict(params)
    params["is_compressed"] = True
    nt = int(params["ntypes"])
    m = om.OracleModel(params | {"is_compressed": False}, variables, torch.float64)
    cv = {}
    for k in range(nt * nt):
        i = k // nt
        mean, std = float(params["sr_mean"][i]), float(params["sr_std"][i])
        lo = (0.0 - mean) / std
        hi = (float(om.sr(torch.tensor(rmin, dtype=torch.float64), float(params["rcut"]))) - mean) / std
        x = torch.linspace(lo, hi, ngrids + 1, dtype=torch.float64).requires_grad_(True)
        f0 = m.embed(k, x)                                  # (ngrids+1, W)
        W = f0.shape[1]
        f1 = torch.stack([torch.autograd.grad(f0[:, w].sum(), x, create_graph=True)[0] for w in range(W)], 1)
        f2 = torch.stack([torch.autograd.grad(f1[:, w].sum(), x, retain_graph=True)[0] for w in range(W)], 1)
        f0, f1, f2 = f0.detach().numpy(), f1.detach().numpy(), f2.detach().numpy()
        h = (hi - lo) / ngrids
        # p(t) = a0 + a1 t + ... + a5 t^5 on [0, h] with end conditions
        M3 = np.array([[h ** 3, h ** 4, h ** 5], [3 * h ** 2, 4 * h ** 3, 5 * h ** 4], [6 * h, 12 * h ** 2, 20 * h ** 3]])
        a0, a1, a2 = f0[:-1], f1[:-1], 0.5 * f2[:-1]
        rhs = np.stack([f0[1:] - (a0 + a1 * h + a2 * h ** 2), f1[1:] - (a1 + 2 * a2 * h), f2[1:] - 2 * a2], 1)
        a345 = np.einsum("ij,njw->niw", np.linalg.inv(M3), rhs)     # (ngrids, 3, W)
        coeff = np.stack([a345[:, 2], a345[:, 1], a345[:, 0], a2, a1, a0], 1)  # x0^5 ... x0^0
        cv["embedding_net_%d" % k] = {"srmin": np.float32(lo), "srmax": np.float32(hi),
                                      "poly_coeff": coeff.astype(np.float32)}
    variables = dict(variables)
    variables["compress_var"] = cv
    return params, variables


def ref_energy_force(ref, params, variables, coord, box3, type_idx, nbrs_nm=None):
    dpmodel = ref["dpmodel"]
    data = ref["data"]
    from jaxshim import J
    model = dpmodel.DPModel(params)
    box33 = np.diag(box3)
    if nbrs_nm is None:
        lattice = data.compute_lattice_candidate(J(box33)[None], params["rcut"], print_info=False)
        static_args = {"type_idx": tuple(int(t) for t in type_idx), "use_neighbor_list": False, "lattice": lattice}
    else:
        static_args = {"type_idx": tuple(int(t) for t in type_idx), "use_neighbor_list": True}
        nbrs_nm = [[J(np.asarray(a, np.int64)) for a in row] for row in nbrs_nm]
    c = J(np.asarray(coord, np.float64)).requires_grad_(True)
    E, _ = model.apply(variables, c, J(box33), static_args, nbrs_nm)
    g = torch.autograd.grad(E, c)[0]
    return float(E), (-g).detach().numpy().astype(np.float64)


def typed_to_nbrs_nm(typed, type_count, sel):
    offs = np.concatenate([[0], np.cumsum(type_count)])
    col = np.concatenate([[0], np.cumsum(sel)])
    return [[typed[offs[i]:offs[i + 1], col[j]:col[j + 1]] for j in range(len(sel))]
            for i in range(len(type_count))]


def golden_models():
    """The three models the fixtures use, rebuilt deterministically:
    A = the benchmark model (random init, zero biases, mean 0 / std 1),
    B = every parameter non-trivial, C = B with a compressed-embedding table."""
    wA = water_box(4, 12.42, seed=0)
    nn = nnbrs_rule(wA["position"], wA["box"], wA["type_idx"], 6.0)
    pA, vA = init_dp_params(nnbrs=nn, seed=0)
    pB, vB = randomize_model(*init_dp_params(nnbrs=nn, seed=1), seed=11)
    pC, vC = compressed_variant(pB, vB, seed=12)
    return {"A": (pA, vA), "B": (pB, vB), "C": (pC, vC)}


def main(ref_root):
    import jaxshim
    ref = jaxshim.load_reference(ref_root)
    sel = [46, 92]
    models = golden_models()
    (pA, vA), (pB, vB), (pC, vC) = models["A"], models["B"], models["C"]

    # --- system A: 192-atom water, lattice (all-pairs) path, benchmark model
    wA = water_box(4, 12.42, seed=0)
    EA, FA = ref_energy_force(ref, pA, vA, wA["position"], wA["box"], wA["type_idx"])
    # --- same system, all-terms-nonzero model
    EB, FB = ref_energy_force(ref, pB, vB, wA["position"], wA["box"], wA["type_idx"])
    # --- compressed branch
    EC, FC = ref_energy_force(ref, pC, vC, wA["position"], wA["box"], wA["type_idx"])

    # --- system D: 1536-atom water, neighbour-list path (box > 2 (rcut + skin))
    wD = water_box(8, 24.83, seed=3)
    cnt = np.bincount(wD["type_idx"], minlength=2)
    c = onl.canonicalize(wD["position"], wD["box"], wD["type_idx"])
    typed, counts, ovf = onl.typed_nlist(c, wD["box"].astype(np.float32), onl.cutoff_sq(6.3), cnt, sel)
    assert not ovf
    ED, FD = ref_energy_force(ref, pB, vB, wD["position"], wD["box"], wD["type_idx"],
                              nbrs_nm=typed_to_nbrs_nm(typed, cnt, sel))

    # --- system E: 96-atom frame in a box smaller than 2 rcut (multiple images)
    wE = water_box(4, 9.86, seed=5, n_water=32)
    EE, FE = ref_energy_force(ref, pB, vB, wE["position"], wE["box"], wE["type_idx"])

    # --- ring-polymer normal modes from pimd.py
    pimd = ref["pimd"]
    kT = 300 * 8.617333e-5
    freqs, C = pimd.normal_mode_transform(8, kT)

    np.savez_compressed(
        os.path.join(HERE, "golden_model.npz"),
        A_pos=wA["position"], A_box=wA["box"], A_type=wA["type_idx"], A_E=EA, A_F=FA,
        B_E=EB, B_F=FB, C_E=EC, C_F=FC,
        D_pos=wD["position"], D_box=wD["box"], D_type=wD["type_idx"], D_E=ED, D_F=FD, D_nbrs=typed,
        E_pos=wE["position"], E_box=wE["box"], E_type=wE["type_idx"], E_E=EE, E_F=FE,
        pimd_freqs=freqs, pimd_C=C)
    print("A", EA, "B", EB, "C", EC, "D", ED, "E", EE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path to the deepmd-jax source checkout>" % os.path.basename(sys.argv[0]))
    main(sys.argv[1])
