"""Shared helpers for the GPU parity tests (call the library through the
C ABI via deepmd_jax_b200.engine)."""
import numpy as np
import torch


def run_gpu(params, variables, positions, box, type_idx, sel=(46, 92), precision="fp32", skin=0.3,
            device_model=None):
    """positions (F,N,3) user order; returns dict of numpy arrays (user order)."""
    from deepmd_jax_b200.engine import DeviceModel, NeighborBuilder, sort_by_type
    dm = device_model or DeviceModel(params, variables)
    positions = np.asarray(positions, dtype=np.float64)
    if positions.ndim == 2:
        positions = positions[None]
    F, N = positions.shape[:2]
    perm, cnt = sort_by_type(type_idx, int(params["ntypes"]))
    pos = torch.tensor(np.ascontiguousarray(positions), dtype=torch.float32, device="cuda").contiguous()
    pm = torch.tensor(perm, dtype=torch.int32, device="cuda")
    boxt = torch.tensor(np.tile(np.asarray(box, np.float32), (F, 1)), device="cuda")
    nb = NeighborBuilder(N, F, cnt, list(sel), box, float(params["rcut"]) + skin)
    nbrs, st = nb.build(pos, perm=pm)
    out = dm.evaluate(pos, boxt, nbrs, cnt, list(sel), perm=pm, precision=precision, atom_energy=True)
    torch.cuda.synchronize()
    return dict(energy=out["energy"].cpu().numpy(), force=out["force"].cpu().numpy(),
                virial=out["virial"].cpu().numpy().reshape(F, 3, 3),
                atom_energy=out["atom_energy"].cpu().numpy(), status=int(out["status"].item()) | int(st.item()),
                nbrs=nbrs.cpu().numpy())
