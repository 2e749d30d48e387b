"""Error table of the FP32 and mixed (BF16 tensor-core) forms against an FP64
evaluation of the same weights: 12,288-atom water (4,096 H2O, L = 49.66 A),
32 frames displaced by N(0, 0.05 A) (seeds 1..32), for the benchmark model
(random init, zero biases) and for a model whose every parameter is
non-trivial.  The FP64 numbers come from the oracle, run in float64 on the
GPU through torch; neighbour lists are the device lists (bit-exact to the
oracle's, tested in test_gpu_nlist.py) at rcut 6.0 A.

Tolerances (the mixed-form target is an RMS force error <= 5e-3 eV/A):
  FP32:  force RMS error <= 1e-4 x force RMS;  energy/atom RMS <= 1e-6 eV + 1e-6 x |E|/N
  mixed: force RMS error <= 5e-3 eV/A and <= 3e-2 x force RMS;
         energy/atom RMS <= 2e-2 x mean |E_atom|;  virial/atom RMS <= 3e-2 x RMS(W/N)
Run with -s to print the table.
"""
import numpy as np
import pytest
import torch

from make_golden import golden_models
from oracle import model as om

pytestmark = pytest.mark.gpu

NF = 32


def _frames():
    from deepmd_jax_b200.systems import water_box
    w = water_box(16, 49.66, seed=0)
    pos = np.stack([w["position"] + np.random.default_rng(s).normal(scale=0.05, size=w["position"].shape)
                    for s in range(1, NF + 1)])
    return w, pos


def _device(p, v, w, pos, precision):
    from deepmd_jax_b200.engine import DeviceModel, NeighborBuilder, sort_by_type
    perm, cnt = sort_by_type(w["type_idx"], 2)
    pm = torch.tensor(perm.astype(np.int32), device="cuda")
    P = torch.tensor(np.ascontiguousarray(pos, dtype=np.float32), device="cuda")
    box = torch.tensor(np.ascontiguousarray(np.broadcast_to(w["box"], (NF, 3)), dtype=np.float32), device="cuda")
    sel = [46, 92]
    nbrs, st = NeighborBuilder(pos.shape[1], NF, cnt, sel, w["box"], 6.0).build(P, perm=pm)
    assert int(st.item()) == 0
    out = DeviceModel(p, v).evaluate(P, box, nbrs, cnt, sel, perm=pm, precision=precision, atom_energy=True)
    assert int(out["status"].item()) == 0
    return ({k: out[k].cpu().numpy() for k in ("energy", "force", "virial", "atom_energy")},
            nbrs.cpu().numpy(), perm, sel)


@pytest.mark.parametrize("mk", ["A", "B"])
def test_error_table_fp32_and_mixed_vs_fp64(mk):
    p, v = golden_models()[mk]
    w, pos = _frames()
    N = pos.shape[1]
    got = {prec: _device(p, v, w, pos, prec) for prec in ("fp32", "mixed")}
    nbrs = got["fp32"][1]
    m64 = om.OracleModel(p, v, torch.float64, device="cuda")
    ref = [om.energy_force(m64, pos[f], w["box"], w["type_idx"], nbrs=nbrs[f], sel=[46, 92]) for f in range(NF)]
    E64 = np.array([r["energy"] for r in ref])
    F64 = np.stack([r["force"] for r in ref])
    W64 = np.stack([r["virial"].reshape(9) for r in ref])
    A64 = np.stack([r["atom_energy"] for r in ref])
    frms = np.sqrt((F64 ** 2).mean())
    wrms = np.sqrt(((W64 / N) ** 2).mean())
    print("\nmodel %s: force RMS %.4e eV/A, |E|/N %.4e eV, virial/N RMS %.4e eV" %
          (mk, frms, np.abs(E64).mean() / N, wrms))
    print("%-6s %14s %14s %14s %14s %14s" % ("form", "E/atom RMS", "E_atom RMS", "F RMS", "F RMS rel", "W/N RMS"))
    for prec, (o, _, _, _) in got.items():
        e_err = np.sqrt((((o["energy"] - E64) / N) ** 2).mean())
        ea_err = np.sqrt(((o["atom_energy"] - A64) ** 2).mean())
        f_err = np.sqrt(((o["force"] - F64) ** 2).mean())
        w_err = np.sqrt((((o["virial"] - W64) / N) ** 2).mean())
        print("%-6s %14.4e %14.4e %14.4e %14.4e %14.4e" % (prec, e_err, ea_err, f_err, f_err / frms, w_err))
        if prec == "fp32":
            assert f_err <= 1e-4 * frms
            assert e_err <= 1e-6 + 1e-6 * np.abs(E64).mean() / N
            assert w_err <= 1e-4 * wrms + 1e-9
        else:
            assert f_err <= 5e-3 and f_err <= 3e-2 * frms
            assert e_err <= 2e-2 * np.abs(A64).mean()
            assert w_err <= 3e-2 * wrms + 1e-9
