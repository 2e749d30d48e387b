"""Drop-in for deepmd_jax.dpmodel.DPModel (deepmd_jax/dpmodel.py:10-108) for
se_a energy models, evaluated by libdpb200 on the GPU.

``DPModel(params).apply(variables, coord_N3, box_33, static_args, nbrs_nm)``
returns ``(energy, debug)`` like the flax module (debug: the descriptor T);
``energy_and_force``
returns ``(energy, force)`` with the force as the negative coordinate
gradient (dpmodel.py:106-108), computed by the hand-written adjoint.

Inputs follow the reference: ``coord_N3`` (N, 3) in the user's atom order,
``box_33`` a (3, 3) box with the lattice vectors as rows (or (3,) / scalar
for an orthorhombic one), ``static_args`` a mapping with ``'type_idx'``;
``nbrs_nm`` the nested typed list of ``md_utils.typed_neighbor_list``
(type-local indices, pad N; orthorhombic boxes) or None, in which case every
periodic image within rcut is summed, as the reference's lattice path does
(deepmd_jax/utils.py:66-78); a general box takes the open ghost-atom system
of ``lattice.ghost_eval``.  Arrays may be numpy or torch;
results are numpy (energy float, force (N, 3) float32).
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import DeviceModel, _require_cuda, sort_by_type
from .lattice import ghost_eval
from .md_utils import exact_neighbor_list, from_nbrs_nm


def general_box(box):
    """The (3, 3) matrix of a (9,) or (3, 3) box with off-diagonal entries,
    else None (orthorhombic boxes take the direct path)."""
    b = np.asarray(box, dtype=np.float64)
    if b.size == 9:
        m = b.reshape(3, 3)
        if np.any(m - np.diag(np.diag(m))):
            return m
    return None


def box_diagonal(box):
    """(3,) orthorhombic box lengths from a scalar, (3,), (9,) or (3, 3) box;
    a box with off-diagonal entries is rejected here (general boxes go
    through lattice.ghost_eval)."""
    b = np.asarray(box, dtype=np.float64)
    if b.size == 1:
        return np.repeat(b.reshape(1), 3)
    if b.size == 3:
        return b.reshape(3)
    if b.size == 9:
        m = b.reshape(3, 3)
        if np.any(m - np.diag(np.diag(m))):
            raise NotImplementedError("non-orthorhombic boxes are not supported by the B200 kernels")
        return np.diag(m).copy()
    raise ValueError("box must be a scalar, (3,), (9,) or (3, 3)")


class DPModel:
    """se_a energy model with the reference DPModel's methods.

    ``precision`` selects 'fp32' (default; the reference's float32) or
    'mixed' (BF16 tensor-core contractions with FP32 accumulation)."""

    def __init__(self, params, precision="fp32"):
        self.params = params
        self.precision = precision
        self._dev = {}

    def _device_model(self, variables):
        key = id(variables)
        hit = self._dev.get(key)
        if hit is None or hit[0] is not variables:
            _require_cuda()
            hit = (variables, DeviceModel(self.params, variables))
            self._dev = {key: hit}
        return hit[1]

    def _run(self, variables, coord_N3, box_33, static_args, nbrs_nm, descriptors=False):
        """{'energy' float, 'force' (N, 3) float32, 'virial' (3, 3), 'T'
        (with ``descriptors``)} of one configuration."""
        dm = self._device_model(variables)
        type_idx = np.asarray(static_args["type_idx"], dtype=int)
        N = len(type_idx)
        nt = int(self.params["ntypes"])
        gb = general_box(box_33)
        if gb is not None:
            if nbrs_nm is not None:
                raise NotImplementedError("a typed neighbour list takes an orthorhombic box (the reference's "
                                          "neighbour-list path uses only the box diagonal)")
            c = coord_N3.detach().cpu().numpy() if torch.is_tensor(coord_N3) else np.asarray(coord_N3)
            r = ghost_eval(dm, c.reshape(N, 3), gb, type_idx, nt, float(self.params["rcut"]), self.precision,
                           virial=True, descriptors=descriptors)
            return r
        perm, count = sort_by_type(type_idx, nt)
        perm_dev = torch.tensor(perm.astype(np.int32), device="cuda")
        c = coord_N3 if torch.is_tensor(coord_N3) else torch.as_tensor(np.asarray(coord_N3))
        pos = c.to(device="cuda", dtype=torch.float32).reshape(1, N, 3).contiguous()
        L = box_diagonal(box_33)
        box = torch.tensor(L[None], dtype=torch.float32, device="cuda")
        if nbrs_nm is None:
            nbrs, sel = exact_neighbor_list(pos, perm_dev, count, L[None], float(self.params["rcut"]))
        else:
            packed, sel = from_nbrs_nm(nbrs_nm)
            if packed.shape[0] != N:
                raise ValueError("nbrs_nm rows (%d) do not match the atom count (%d)" % (packed.shape[0], N))
            nbrs = packed[None].contiguous()
        out = dm.evaluate(pos, box, nbrs, count, sel, perm=perm_dev, precision=self.precision)
        st = int(out["status"].item())
        if st & 2:
            raise RuntimeError("neighbour list overflow (status %d): reallocate the typed neighbour list" % st)
        res = {"energy": float(out["energy"][0].item()), "force": out["force"][0].cpu().numpy(),
               "virial": out["virial"][0].cpu().numpy().reshape(3, 3)}
        if descriptors:
            T, _ = dm.descriptors(pos, box, nbrs, count, sel, perm=perm_dev, precision=self.precision)
            res["T"] = T.cpu().numpy()
        return res

    def apply(self, variables, coord_N3, box_33, static_args, nbrs_nm=None):
        """(energy, debug) like the flax module: debug is the descriptor
        T_NselXW (N, 10, W), T / Nnbrs without Tbias, atoms in type-sorted
        order (deepmd_jax/dpmodel.py:50-51,99-100)."""
        out = self._run(variables, coord_N3, box_33, static_args, nbrs_nm, descriptors=True)
        return out["energy"], out["T"]

    def energy(self, variables, coord_N3, box_33, static_args, nbrs_nm=None):
        return self._run(variables, coord_N3, box_33, static_args, nbrs_nm)["energy"]

    def energy_and_force(self, variables, coord_N3, box_33, static_args, nbrs_nm=None):
        out = self._run(variables, coord_N3, box_33, static_args, nbrs_nm)
        return out["energy"], out["force"]

    def energy_force_virial(self, variables, coord_N3, box_33, static_args, nbrs_nm=None):
        """Energy, force and the 3x3 virial W = -sum_ij r_ij (x) f_ij, whose
        trace is -dU/d(eps) of the reference's perturbation derivative
        (deepmd_jax/md.py:416-444, routine.py:265-273)."""
        out = self._run(variables, coord_N3, box_33, static_args, nbrs_nm)
        return out["energy"], out["force"], out["virial"]


class EnergyFunction(torch.autograd.Function):
    """E(coord) as a torch autograd node whose backward is the hand-written
    adjoint (grad = -force); used for gradient checks, not on the MD path.

    ``EnergyFunction.apply(coord, model, variables, box, type_idx)`` with
    ``coord`` (N, 3) float64/float32 (any device) returns the energy as a
    0-d float64 tensor on coord's device."""

    @staticmethod
    def forward(ctx, coord, model, variables, box, type_idx):
        e, f = model.energy_and_force(variables, coord.detach(), box, {"type_idx": tuple(type_idx)})
        ctx.save_for_backward(torch.as_tensor(f, dtype=coord.dtype, device=coord.device))
        return torch.tensor(e, dtype=torch.float64, device=coord.device)

    @staticmethod
    def backward(ctx, g):
        (f,) = ctx.saved_tensors
        return -f * g.to(f.dtype), None, None, None, None
