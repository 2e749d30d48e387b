"""Serving loop (deepmd_jax_b200.serving.Server) on the GPU: requests of
different atom counts, frame counts and boxes (a 96-atom box below 2 rcut
included) evaluated in packed batches, with an MD-continuation request
stepping beside them, must give what each request gives alone.

Tolerances: the packed batch runs the same per-atom arithmetic as the request
alone; only the order of float atomics differs.  Energy |dE| <= 1e-9 |E| +
1e-9 eV, forces and virial max diff <= 1e-5 of their max (both forms).  The
MD request after 20 NVT steps: positions within 1e-4 A of the same run alone.
"""
import numpy as np
import pytest
import torch

from make_golden import golden_models
from oracle import model as om

pytestmark = pytest.mark.gpu


def _systems():
    from deepmd_jax_b200.systems import water_box
    rng = np.random.default_rng(5)
    out = []
    w = water_box(4, 12.42, seed=1)                         # 192 atoms, 3 frames, one box
    out.append((np.stack([w["position"] + rng.normal(scale=0.03, size=w["position"].shape) for _ in range(3)]),
                np.array(w["box"]), w["type_idx"]))
    w = water_box(4, 9.86, seed=2, n_water=32)              # 96 atoms, small box (images)
    out.append((np.stack([w["position"], w["position"] + 0.1]), np.array(w["box"]), w["type_idx"]))
    w = water_box(8, 24.83, seed=3)                         # 1,536 atoms
    out.append((w["position"][None], np.array(w["box"]), w["type_idx"]))
    w = water_box(4, 12.42, seed=4)                         # 192 atoms, two frames with different boxes
    order = rng.permutation(192)                            # atoms not sorted by type
    out.append((np.stack([w["position"][order], w["position"][order] * 1.02]),
                np.stack([w["box"], w["box"] * 1.02]), w["type_idx"][order]))
    return out


def _alone(dm, coord, box, type_idx, precision):
    from deepmd_jax_b200.engine import NeighborBuilder, sort_by_type
    F, N = coord.shape[:2]
    boxes = np.broadcast_to(np.asarray(box, np.float32).reshape(-1, 3), (F, 3))
    perm, cnt = sort_by_type(type_idx, 2)
    pm = torch.tensor(perm.astype(np.int32), device="cuda")
    E, Fo, W = [], [], []
    for f in range(F):
        pos = torch.tensor(np.ascontiguousarray(coord[f:f + 1], dtype=np.float32), device="cuda")
        nbrs, _ = NeighborBuilder(N, 1, cnt, [46, 92], boxes[f], 6.0).build(pos, perm=pm)
        bx = torch.tensor(np.ascontiguousarray(boxes[f:f + 1]), device="cuda")
        o = dm.evaluate(pos, bx, nbrs, cnt, [46, 92], perm=pm, precision=precision)
        E.append(float(o["energy"][0]))
        Fo.append(o["force"][0].cpu().numpy())
        W.append(o["virial"][0].cpu().numpy().reshape(3, 3))
    return np.array(E), np.stack(Fo), np.stack(W)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_packed_batches_match_requests_alone(precision):
    from deepmd_jax_b200.engine import DeviceModel
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.serving import Server
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["B"]
    systems = _systems()
    wmd = water_box(4, 12.42, seed=9)
    with Server((p, v), precision=precision, hbm_budget=8e9) as srv:
        fmd = srv.submit_md(wmd["position"], wmd["box"], wmd["type_idx"], wmd["mass_per_type"], 20, routine="NVT",
                            velocity=wmd["velocity"], seed=3)
        futs = [srv.submit_evaluate(c, b, t) for c, b, t in systems]
        res = [f.result(timeout=300) for f in futs]
        md = fmd.result(timeout=300)
        lat = srv.latency_summary()
    assert lat["eval"]["n"] == len(systems) and lat["md"]["n"] == 1
    dm = DeviceModel(p, v)
    for (c, b, t), r in zip(systems, res):
        assert r["status"] == 0
        E, F, W = _alone(dm, c, b, t, precision)
        assert np.all(np.abs(r["energy"] - E) <= 1e-9 * np.abs(E) + 1e-9), (r["energy"], E)
        assert np.abs(r["force"] - F).max() <= 1e-5 * np.abs(F).max()
        assert np.abs(r["virial"] - W).max() <= 1e-5 * np.abs(W).max()
    if precision == "fp32":                              # one request against the float64 oracle too
        c, b, t = systems[1]
        ref = om.energy_force(om.OracleModel(p, v, torch.float64), c[0], b, t)
        assert abs(res[1]["energy"][0] - ref["energy"]) <= 2e-6 * np.abs(ref["atom_energy"]).sum() + 1e-6
        assert np.abs(res[1]["force"][0] - ref["force"]).max() <= 2e-4 * np.abs(ref["force"]).max()
    sim = Simulation((p, v), wmd["box"], wmd["type_idx"], wmd["mass_per_type"], "NVT", 0.5, wmd["position"],
                     initial_velocity=wmd["velocity"], temperature=300.0, seed=3, report_interval=10,
                     precision=precision, verbose=False)
    sim.run(20, trajectory=False)
    assert np.abs(md["position"] - sim.getPosition()).max() < 1e-4


def test_admission_waits_for_the_budget():
    """With a budget that holds one request at a time every request still
    completes and the reserved bytes never exceed the budget."""
    from deepmd_jax_b200.serving import Server
    from deepmd_jax_b200.systems import water_box
    p, v = golden_models()["B"]
    w = water_box(8, 24.83, seed=3)
    one = Server((p, v)).eval_bytes(len(w["type_idx"]))
    with Server((p, v), hbm_budget=int(1.5 * one)) as srv:
        futs = [srv.submit_evaluate(w["position"] + 0.01 * k, w["box"], w["type_idx"]) for k in range(4)]
        res = [f.result(timeout=300) for f in futs]
        assert srv.budget.peak <= srv.budget.total
        assert srv.batches == 4
        with pytest.raises(ValueError):
            srv.submit_evaluate(np.stack([w["position"]] * 4), w["box"], w["type_idx"])
    assert all(np.isfinite(r["energy"]).all() and r["status"] == 0 for r in res)
