"""ORACLE (test infrastructure only): CPU restatement of deepmd-jax's se_a
energy model, used by the tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` as the checker.  It is never part of the product path.

Everything here is written with torch tensors so one code path runs in float64
(the parity reference, forces by autograd) and float32 (the CPU baseline).

Restated from the reference source:
  * ``sr`` ............................ deepmd_jax/utils.py:29-32
  * ``shift`` (orthorhombic) .......... deepmd_jax/utils.py:20-27
  * ``tensor_3to6`` ................... deepmd_jax/utils.py:51-52
  * relative coordinates ............... deepmd_jax/utils.py:54-87
  * env matrix + normalisation ........ deepmd_jax/dpmodel.py:36-47
  * embedding net (uncompressed) ...... deepmd_jax/utils.py:100-125
  * embedding net (compressed) ........ deepmd_jax/utils.py:126-151
  * descriptor T, Tbias, G ............ deepmd_jax/dpmodel.py:50-51,73-78
  * fitting net + Ebias + sum ......... deepmd_jax/utils.py:153-166, dpmodel.py:79-81
  * forces = -dE/dcoord ............... deepmd_jax/dpmodel.py:106-108

Parity status: the model arithmetic is pinned against golden vectors produced
by running the reference's own ``dpmodel.py``/``utils.py`` source through a
torch-backed stand-in for jax/flax (tests/golden/make_golden.py).  The
neighbour-list construction lives in the third-party jax_md package, which is
absent here; its restatement (oracle/nlist.py) is parity-unpinned at the
one-ulp boundary of the cutoff test.
"""
from __future__ import annotations

import math
import numpy as np
import torch

SQRT2 = math.sqrt(2.0)
SQRT3 = math.sqrt(3.0)


def sr(r, rcut):
    """1/r with the reference's smooth cutoff (utils.py:29-32)."""
    t = r / rcut
    mask = ((r > 1e-14) & (t < 1)).to(r.dtype)
    return mask / (r + 1e-15) * (1 - 3 * t ** 2 + 2 * t ** 3)


def tensor_3to6(x, axis, bias=0.0):
    """[x^2 - bias, sqrt2 * x * roll(x, 1)] along ``axis`` (utils.py:51-52)."""
    return torch.cat([x ** 2 - bias, SQRT2 * x * torch.roll(x, shifts=1, dims=axis)], dim=axis)


def shift_ortho(d, box3):
    """(d - L/2) mod L - L/2 with python-style mod (utils.py:24-26)."""
    return torch.remainder(d - box3 / 2, box3) - box3 / 2


def _t(a, dtype, device="cpu"):
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=device)


class OracleModel:
    """Holds one model's parameters as torch tensors of a chosen dtype."""

    def __init__(self, params, variables, dtype=torch.float64, device="cpu"):
        self.params = params
        self.dtype = dtype
        self.device = torch.device(device)

        def _td(a, dt):
            return _t(a, dt, self.device)

        v = variables["params"]
        p = params
        self.nt = int(p["ntypes"])
        self.rcut = float(p["rcut"])
        self.A = int(p["axis"])
        self.ew = list(p["embed_widths"])
        self.fw = list(p["fit_widths"])
        self.mean = _td(p["sr_mean"], dtype)
        self.std = _td(p["sr_std"], dtype)
        self.nnbrs = float(p["Nnbrs"])
        self.ebias = _td(p["Ebias"], dtype)
        self.out_norm = float(p.get("out_norm", 1.0))
        self.compressed = bool(p.get("is_compressed", False))
        self.emb = []
        for k in range(self.nt * self.nt):
            net = v["embedding_net_%d" % k]
            self.emb.append([(_td(net["Dense_%d" % i]["kernel"], dtype), _td(net["Dense_%d" % i]["bias"], dtype))
                             for i in range(len(self.ew))])
        self.tbias = _td(v["Tbias"], dtype)
        self.fit = []
        for t in range(self.nt):
            net = v["fitting_net_%d" % t]
            layers = []
            for i in range(len(self.fw) + 1):
                d = net["Dense_%d" % i]
                dt = net.get("dt%d" % i) if 0 < i < len(self.fw) else None
                layers.append((_td(d["kernel"], dtype), _td(d["bias"], dtype),
                               None if dt is None else _td(dt, dtype)))
            self.fit.append(layers)
        self.cvar = None
        if self.compressed:
            cv = variables["compress_var"]
            self.cvar = [(float(np.asarray(cv["embedding_net_%d" % k]["srmin"])),
                          float(np.asarray(cv["embedding_net_%d" % k]["srmax"])),
                          _td(cv["embedding_net_%d" % k]["poly_coeff"], dtype))
                         for k in range(self.nt * self.nt)]

    # -- embedding net (utils.py:100-151) ---------------------------------
    def embed(self, k, s):
        """s: (...,) normalised s(r) -> (..., W)."""
        if self.compressed:
            srmin, srmax, coeff = self.cvar[k]
            ng = coeff.shape[0]
            delta = (srmax - srmin) / ng
            x = s - srmin
            idx = (x / delta).to(torch.int64)   # astype(int) truncates toward zero
            x0 = x - idx.to(x.dtype) * delta
            # jax gathers clamp out-of-range indices; x0 keeps the unclamped idx
            c = coeff[idx.clamp(0, ng - 1)]
            return sum(c[..., i, :] * x0[..., None] ** (5 - i) for i in range(6))
        x = s[..., None]
        layers = self.emb[k]
        for i, (Wk, b) in enumerate(layers):
            if i == 0:
                x = torch.tanh(x @ Wk + b)
            else:
                # utils.py:115-117: repeat(x, Z) for a widening layer, the mean
                # over the 1/Z groups of reshape(..., 1/Z, width) for a narrowing one
                n_in, n_out = Wk.shape
                if n_out % n_in == 0:
                    x_prev = torch.repeat_interleave(x, n_out // n_in, dim=-1)
                else:
                    x_prev = x.reshape(x.shape[:-1] + (n_in // n_out, n_out)).mean(-2)
                x = torch.tanh(x @ Wk + b) + x_prev
        return x

    # -- fitting net (utils.py:153-166) -------------------------------------
    def fitting(self, t, G):
        x = G
        layers = self.fit[t]
        for i in range(len(self.fw)):
            Wk, b, dt = layers[i]
            x_prev = x
            x = torch.tanh(x @ Wk + b)
            if dt is not None:
                x = x * dt + x_prev
        Wk, b, _ = layers[-1]
        return (x @ Wk + b)[..., 0]

    # -- full model on the slot representation -------------------------------
    def atomic_energy(self, x_groups, valid_groups, type_count):
        """Per-atom energies.

        x_groups[j]: (N, S_j, 3) relative coordinates (neighbour - centre) for
        neighbour type j, centres in type-sorted order; valid_groups[j]: (N, S_j)
        bool.  type_count: atoms per type (centres are sorted by type).
        Returns (E_atom (N,), T (N,10,W)).
        """
        dtype = self.dtype
        N = x_groups[0].shape[0]
        dev = x_groups[0].device
        ctype = torch.repeat_interleave(torch.arange(self.nt, device=dev), torch.as_tensor(type_count, device=dev))
        mean = self.mean[ctype]
        std = self.std[ctype]
        W = self.ew[-1]
        T = torch.zeros((N, 10, W), dtype=dtype, device=dev)
        for j in range(self.nt):
            x = x_groups[j]
            valid = valid_groups[j].to(dtype)
            xg = torch.where(x.abs() > 1e-15, x, torch.full_like(x, 1e-15))
            r = torch.linalg.norm(xg, dim=-1) * valid
            x = x * valid[..., None]
            s = sr(r, self.rcut)
            sn = s / std[:, None]
            st = (s - mean[:, None]) / std[:, None]
            xh = x / (r + 1e-16)[..., None]
            R3 = SQRT3 * sn[..., None] * xh
            R6 = 3 * sn[..., None] * tensor_3to6(xh, -1, 1.0 / 3.0)
            Rt = torch.cat([sn[..., None], R3, R6], dim=-1)   # (N, S, 10)
            off = 0
            for i in range(self.nt):
                n_i = int(type_count[i])
                if n_i == 0 or x.shape[1] == 0:
                    off += n_i
                    continue
                e = self.embed(i * self.nt + j, st[off:off + n_i])       # (n_i, S, W)
                T[off:off + n_i] = T[off:off + n_i] + torch.einsum("nsc,nsw->ncw", Rt[off:off + n_i], e)
                off += n_i
        T = T / self.nnbrs
        A = self.A
        T0 = T[:, 0] + self.tbias
        T3 = T[:, 1:4]
        T6 = T[:, 4:]
        G = T0[:, None, :] * T0[:, :A, None] + (T3[:, :, None, :] * T3[:, :, :A, None]).sum(1)
        G2 = tensor_3to6(T3[:, :, A:2 * A], 1) + T6[:, :, A:2 * A]
        G = G + (G2[..., None] * T6[:, :, None, :]).sum(1)
        G = G.reshape(N, -1)
        E = torch.zeros(N, dtype=dtype, device=dev)
        off = 0
        for i in range(self.nt):
            n_i = int(type_count[i])
            if n_i:
                E[off:off + n_i] = (self.fitting(i, G[off:off + n_i]) + self.ebias[i]) * self.out_norm
            off += n_i
        return E, T


def sort_by_type(type_idx, ntypes):
    type_idx = np.asarray(type_idx)
    perm = np.argsort(type_idx, kind="stable")
    count = np.bincount(type_idx, minlength=ntypes)
    return perm, count


def relative_coords_nlist(coord_sorted, box3, nbrs, sel, type_count):
    """Neighbour-list branch of get_relative_coord (utils.py:79-82).

    nbrs: (N, sum(sel)) int array in the typed block layout: columns
    [off_j, off_j + sel_j) hold type-local indices of type-j neighbours,
    padding = N.  Returns per-type (x (N,S_j,3), valid (N,S_j))."""
    N = coord_sorted.shape[0]
    offs = np.concatenate([[0], np.cumsum(type_count)])
    col = np.concatenate([[0], np.cumsum(sel)])
    xs, vs = [], []
    for j in range(len(sel)):
        idx = torch.as_tensor(np.asarray(nbrs[:, col[j]:col[j + 1]], dtype=np.int64), device=coord_sorted.device)
        nj = int(type_count[j])
        valid = idx < nj
        cj = coord_sorted[offs[j]:offs[j + 1]]
        if nj == 0:
            xs.append(torch.zeros((N, idx.shape[1], 3), dtype=coord_sorted.dtype, device=coord_sorted.device))
            vs.append(torch.zeros((N, idx.shape[1]), dtype=torch.bool, device=coord_sorted.device))
            continue
        g = cj[idx.clamp(max=nj - 1)]
        x = shift_ortho(g - coord_sorted[:, None, :], box3)
        xs.append(x)
        vs.append(valid)
    return xs, vs


def lattice_images(box3, rcut):
    """Lattice translations whose images can lie within rcut
    (the orthorhombic case of compute_lattice_candidate, data.py:347-364)."""
    n = np.ceil(rcut / np.asarray(box3, float) - 0.5).astype(int)
    g = [np.arange(-k, k + 1) for k in n]
    return np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3)


def relative_coords_lattice(coord_sorted, box3, type_count, rcut):
    """Lattice (all-pairs x images) branch of get_relative_coord (utils.py:66-78)
    for orthorhombic boxes: every atom of type j and every lattice image within
    reach is a slot; images beyond rcut carry s = 0."""
    offs = np.concatenate([[0], np.cumsum(type_count)])
    imgs = torch.as_tensor(lattice_images(box3.detach().cpu().numpy() if torch.is_tensor(box3) else box3, rcut),
                           dtype=coord_sorted.dtype, device=coord_sorted.device) * box3
    xs, vs = [], []
    N = coord_sorted.shape[0]
    for j in range(len(type_count)):
        cj = coord_sorted[offs[j]:offs[j + 1]]
        x = shift_ortho(cj[None, :, :] - coord_sorted[:, None, :], box3)    # (N, M, 3)
        x = (x[:, :, None, :] - imgs[None, None]).reshape(N, -1, 3)
        xs.append(x)
        vs.append(torch.ones(x.shape[:2], dtype=torch.bool, device=x.device))
    return xs, vs


def energy_force(model: OracleModel, coord, box3, type_idx, nbrs=None, sel=None, virial=True):
    """Energy, per-atom energy, forces (user atom order) and virial.

    With ``nbrs`` the neighbour-list path is used (typed block layout); without
    it, the all-pairs lattice path.  The virial is
    W_ab = -sum_pairs x_a dE/dx_b (its trace is -dU/deps under a uniform
    scaling of coordinates and box, md_utils.py:139-159)."""
    dtype = model.dtype
    dev = model.device
    coord = torch.as_tensor(np.asarray(coord), dtype=dtype, device=dev).clone().requires_grad_(True)
    box3 = torch.as_tensor(np.asarray(box3), dtype=dtype, device=dev)
    perm, count = sort_by_type(type_idx, model.nt)
    cs = coord[torch.as_tensor(perm, device=dev)]
    if nbrs is not None:
        xs, vs = relative_coords_nlist(cs, box3, nbrs, sel, count)
    else:
        xs, vs = relative_coords_lattice(cs, box3, count, model.rcut)
    xs_leaf = [x.detach().clone().requires_grad_(True) for x in xs]
    # energy as a function of the relative coordinates; chain to coord below
    E_atom, _ = model.atomic_energy(xs_leaf, vs, count)
    E = E_atom.sum()
    # a type block with no atoms (or no pair slots) does not enter E: zero gradient
    gx = torch.autograd.grad(E, xs_leaf, allow_unused=True)
    gx = [torch.zeros_like(x) if g is None else g for g, x in zip(gx, xs_leaf)]
    # dE/dcoord = sum over slots of gx * dx/dcoord  (x = shift(c_j - c_i))
    used = [(x, g) for x, g in zip(xs, gx) if x.requires_grad]  # empty blocks carry no graph
    gc = (torch.autograd.grad([x for x, _ in used], coord, grad_outputs=[g for _, g in used], allow_unused=True)[0]
          if used else None)
    F = -(torch.zeros_like(coord) if gc is None else gc)
    Wv = None
    if virial:
        Wv = torch.zeros((3, 3), dtype=dtype, device=dev)
        for x, g, v in zip(xs, gx, vs):
            Wv = Wv - torch.einsum("nsa,nsb->ab", x.detach() * v[..., None], g)
    E_user = torch.empty_like(E_atom)
    E_user[torch.as_tensor(perm, device=dev)] = E_atom.detach()
    return dict(energy=float(E.detach()), atom_energy=E_user.cpu().numpy(),
                force=F.detach().cpu().numpy(), virial=None if Wv is None else Wv.cpu().numpy())


def energy_only(model: OracleModel, coord, box3, type_idx, nbrs=None, sel=None):
    dev = model.device
    coord = torch.as_tensor(np.asarray(coord), dtype=model.dtype, device=dev)
    box3 = torch.as_tensor(np.asarray(box3), dtype=model.dtype, device=dev)
    perm, count = sort_by_type(type_idx, model.nt)
    cs = coord[torch.as_tensor(perm, device=dev)]
    if nbrs is not None:
        xs, vs = relative_coords_nlist(cs, box3, nbrs, sel, count)
    else:
        xs, vs = relative_coords_lattice(cs, box3, count, model.rcut)
    with torch.no_grad():
        E_atom, T = model.atomic_energy(xs, vs, count)
    return float(E_atom.sum()), E_atom, T
