"""``evaluate()`` and ``test()`` with the reference's signatures and results
(deepmd_jax/train.py:703-788 and 523-701), evaluated by libdpb200 on the GPU.

The reference writes the frames to a temporary dataset and runs ``test()``
(train.py:523-701), a ``jit(vmap(energy_and_force))`` over ``batch_size``
frames on the lattice path.  Here each batch of frames is one dpb_eval call
over device neighbour lists built at exactly the largest per-type count;
every periodic image within rcut is summed, as on the lattice path
(deepmd_jax/utils.py:66-78).  Training is not part of this library.
"""
from __future__ import annotations

from glob import glob

import numpy as np
import torch

from .engine import DeviceModel, _require_cuda, sort_by_type
from .lattice import ghost_eval
from .md_utils import exact_neighbor_list
from .utils import load_model

_SHAPE_MSG = ('Input shapes are incorrect: \n' +
              'coord: (n_frames, n_atoms, 3) \n' +
              'box: (n_frames) + (,) or (1,) or (3,) or (9), or (3,3) \n' +
              'type_idx (n_atoms).')


def normalize_boxes(coord, box, type_idx):
    """(F, 3, 3) boxes from the shapes evaluate() accepts (train.py:718-740);
    ValueError with the reference's message otherwise."""
    try:
        assert coord.ndim == 3 and coord.shape[2] == 3
        assert type_idx.ndim == 1 and box.ndim in [1, 2, 3]
        assert coord.shape[1] == type_idx.shape[0]
        assert coord.shape[0] == box.shape[0]
        if box.ndim == 1:
            box = box[:, None, None] * np.eye(3)
        elif box.ndim == 2:
            if box.shape[1] == 1:
                box = box[:, None] * np.eye(3)
            elif box.shape[1] == 3:
                box = np.stack([np.diag(b) for b in box])
            else:
                box = box.reshape(box.shape[0], 3, 3)
        elif box.ndim == 3:
            assert box.shape[1] == 3 and box.shape[2] == 3
    except Exception:
        raise ValueError(_SHAPE_MSG)
    return np.asarray(box, dtype=np.float64)


def _map_chemical_types(params, type_idx):
    ct = params.get("chemical_types")
    if ct is None:
        return type_idx
    z = np.array(type_idx, dtype=int)
    unknown = set(z.tolist()) - set(ct)
    if unknown:
        raise ValueError('Atomic numbers %s in type_idx are not in model.params["chemical_types"]=%s'
                         % (sorted(unknown), ct))
    z_to_idx = {zz: i for i, zz in enumerate(ct)}
    return np.array([z_to_idx[zz] for zz in z], dtype=int)


_MODEL_CACHE = {}


def _device_model(model_path):
    hit = _MODEL_CACHE.get(model_path)
    if hit is None:
        model, variables = load_model(model_path, replicate=False)
        if model.params.get("type", "energy") != "energy":
            raise NotImplementedError("evaluate(): only 'energy' models run on libdpb200 (got %r)"
                                      % model.params.get("type"))
        hit = (model, DeviceModel(model.params, variables))
        _MODEL_CACHE.clear()
        _MODEL_CACHE[model_path] = hit
    return hit


def evaluate(model_path, coord, box, type_idx, batch_size=1, precision="fp32"):
    """Energies and forces of frames sharing ``type_idx``.

    coord (n_frames, n_atoms, 3); box (n_frames,) / (n_frames, 1) /
    (n_frames, 3) / (n_frames, 9) / (n_frames, 3, 3), general boxes with the
    lattice vectors as rows included; type_idx
    (n_atoms,) (atomic numbers when the model carries ``chemical_types``).
    Returns {'energy': (n_frames,) float64, 'force': (n_frames, n_atoms, 3)
    float32}, forces in the input atom order.  ``precision`` is 'fp32' (the
    reference's arithmetic) or 'mixed'."""
    coord = np.asarray(coord)
    box = np.asarray(box)
    type_idx = np.asarray(type_idx)
    box = normalize_boxes(coord, box, type_idx)
    _require_cuda()
    model, dm = _device_model(model_path)
    type_idx = _map_chemical_types(model.params, type_idx)
    return _evaluate_frames(model, dm, coord, box, type_idx, batch_size, precision)


def _evaluate_frames(model, dm, coord, box, type_idx, batch_size, precision):
    """Energies and forces of frames (F, N, 3) in boxes (F, 3, 3) with model
    type indices type_idx (N,), batch_size frames per dpb_eval call.  Frames
    in general (non-orthorhombic) boxes are evaluated one at a time through
    their open ghost-atom system (lattice.ghost_eval)."""
    off = box - np.einsum("fii->fi", box)[:, :, None] * np.eye(3)
    general = np.any(off.reshape(len(box), -1) != 0, axis=1)
    L = np.einsum("fii->fi", box)
    F, N = coord.shape[0], coord.shape[1]
    nt = int(model.params["ntypes"])
    perm, count = sort_by_type(type_idx, nt)
    perm_dev = torch.tensor(perm.astype(np.int32), device="cuda")
    rcut = float(model.params["rcut"])
    energy = np.empty(F, dtype=np.float64)
    force = np.empty((F, N, 3), dtype=np.float32)
    for f in np.nonzero(general)[0]:
        r = ghost_eval(dm, coord[f], box[f], type_idx, nt, rcut, precision)
        energy[f], force[f] = r["energy"], r["force"]
    bs = max(int(batch_size), 1)
    ortho = np.nonzero(~general)[0]
    runs, i = [], 0                     # runs of at most bs consecutive orthorhombic frames
    while i < len(ortho):
        j = i + 1
        while j < len(ortho) and j - i < bs and ortho[j] == ortho[j - 1] + 1:
            j += 1
        runs.append((int(ortho[i]), int(ortho[j - 1]) + 1))
        i = j
    for a, b in runs:
        pos = torch.tensor(np.ascontiguousarray(coord[a:b], dtype=np.float32), device="cuda")
        nbrs, sel = exact_neighbor_list(pos, perm_dev, count, L[a:b], rcut)
        bx = torch.tensor(np.ascontiguousarray(L[a:b], dtype=np.float32), device="cuda")
        out = dm.evaluate(pos, bx, nbrs, count, sel, perm=perm_dev, precision=precision)
        energy[a:b] = out["energy"].cpu().numpy()
        force[a:b] = out["force"].cpu().numpy()
    return {"energy": energy, "force": force}


def _flatten_paths(paths):
    for p in paths:
        if isinstance(p, (list, tuple)):
            yield from _flatten_paths(p)
        else:
            yield p


def load_dp_data(data_path):
    """The energy labels of DeepMD-format directories, one entry per
    directory: type.raw and set.*/{coord,box,energy,force}.npy concatenated
    over the sorted sets (deepmd_jax/data.py:22-70,190-200).  type.raw holds
    model type indices.  Extended-XYZ files need ase (data.py:285-345),
    which this library does not use: NotImplementedError."""
    paths = [data_path] if isinstance(data_path, str) else list(_flatten_paths(data_path))
    leaves = []
    for p in paths:
        if isinstance(p, str) and p.lower().endswith((".xyz", ".extxyz")):
            raise NotImplementedError("extxyz datasets are not supported; convert them to DeepMD directories")
        type_idx = np.atleast_1d(np.genfromtxt(p + "/type.raw").astype(int))
        sets = sorted(glob(p + "/set.*/"))
        if not sets:
            raise FileNotFoundError("no set.*/ directory under %r" % p)
        data = {l: np.concatenate([np.load(s + l + ".npy") for s in sets]) for l in ("coord", "box", "energy", "force")}
        nf = len(data["coord"])
        for l, v in data.items():
            assert v.shape[0] == nf, f"{l}.npy has {v.shape[0]} frames, expected {nf}"
        leaves.append({"type_idx": type_idx,
                       "coord": data["coord"].reshape(nf, -1, 3),
                       "box": data["box"].reshape(-1, 3, 3),
                       "energy": data["energy"].reshape(-1),
                       "force": data["force"].reshape(nf, -1, 3)})
    return leaves


def error_metrics(results):
    """RMSE / MAE / l1_mixed of energy per atom and of force components over
    test results (deepmd_jax/train.py:629-690): dE = (E_pred - E_true) / N;
    force RMSE and MAE over all components; l1_mixed force = the mean over
    atoms of each atom's RMS component error."""
    e_sq = e_abs = f_sq = f_abs = f_l1 = 0.0
    e_n = f_n = f_atoms = 0
    for r in results:
        n = len(r["type_idx"])
        dE = (r["predicted_energy"] - r["true_energy"]) / n
        e_sq += dE * dE
        e_abs += abs(dE)
        e_n += 1
        dF = np.asarray(r["predicted_force"], dtype=np.float64) - np.asarray(r["true_force"], dtype=np.float64)
        f_sq += float((dF ** 2).sum())
        f_abs += float(np.abs(dF).sum())
        f_n += dF.size
        f_l1 += float(np.sqrt((dF ** 2).mean(-1)).sum())
        f_atoms += dF.shape[0]
    return {"rmse": {"energy": float(np.sqrt(e_sq / e_n)), "force": float(np.sqrt(f_sq / f_n))},
            "mae": {"energy": float(e_abs / e_n), "force": float(f_abs / f_n)},
            "l1_mixed": {"energy": float(e_abs / e_n), "force": float(f_l1 / f_atoms)}}


def test(model_path, data_path, batch_size=1, precision="fp32"):
    """Errors of an energy model on labelled DeepMD-format data
    (deepmd_jax/train.py:523-701): returns (error_metrics, test_results),
    the results one dict per frame in dataset order with 'box' (3, 3),
    'type_idx', 'predicted_energy', 'true_energy', 'predicted_force',
    'true_force'.  Frames run batch_size at a time through dpb_eval."""
    _require_cuda()
    model, dm = _device_model(model_path)
    results = []
    for leaf in load_dp_data(data_path):
        pred = _evaluate_frames(model, dm, leaf["coord"], np.asarray(leaf["box"], dtype=np.float64),
                                leaf["type_idx"], batch_size, precision)
        for i in range(len(leaf["energy"])):
            results.append({"box": np.asarray(leaf["box"][i]).copy(), "type_idx": leaf["type_idx"].copy(),
                            "predicted_energy": float(pred["energy"][i]), "true_energy": float(leaf["energy"][i]),
                            "predicted_force": pred["force"][i].copy(),
                            "true_force": np.asarray(leaf["force"][i]).copy()})
    return error_metrics(results), results
