"""``evaluate()`` with the reference's signature and results
(deepmd_jax/train.py:703-788), evaluated by libdpb200 on the GPU.

The reference writes the frames to a temporary dataset and runs ``test()``
(train.py:523-701), a ``jit(vmap(energy_and_force))`` over ``batch_size``
frames on the lattice path.  Here each batch of frames is one dpb_eval call
over device neighbour lists built at exactly the largest per-type count;
every periodic image within rcut is summed, as on the lattice path
(deepmd_jax/utils.py:66-78).  Training is not part of this library.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import DeviceModel, _require_cuda, sort_by_type
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
    (n_frames, 3) / (n_frames, 9) / (n_frames, 3, 3), orthorhombic; type_idx
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
    off = box - np.einsum("fii->fi", box)[:, :, None] * np.eye(3)
    if np.any(off):
        raise NotImplementedError("non-orthorhombic boxes are not supported by the B200 kernels")
    L = np.einsum("fii->fi", box)
    F, N = coord.shape[0], coord.shape[1]
    nt = int(model.params["ntypes"])
    perm, count = sort_by_type(type_idx, nt)
    perm_dev = torch.tensor(perm.astype(np.int32), device="cuda")
    rcut = float(model.params["rcut"])
    energy = np.empty(F, dtype=np.float64)
    force = np.empty((F, N, 3), dtype=np.float32)
    bs = max(int(batch_size), 1)
    for a in range(0, F, bs):
        b = min(a + bs, F)
        pos = torch.tensor(np.ascontiguousarray(coord[a:b], dtype=np.float32), device="cuda")
        nbrs, sel = exact_neighbor_list(pos, perm_dev, count, L[a:b], rcut)
        bx = torch.tensor(np.ascontiguousarray(L[a:b], dtype=np.float32), device="cuda")
        out = dm.evaluate(pos, bx, nbrs, count, sel, perm=perm_dev, precision=precision)
        energy[a:b] = out["energy"].cpu().numpy()
        force[a:b] = out["force"].cpu().numpy()
    return {"energy": energy, "force": force}
