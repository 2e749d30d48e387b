"""Device-side engine: a model uploaded through the C ABI, typed neighbour
lists and batched energy/force/virial evaluation on torch CUDA tensors.

torch provides device memory and the current CUDA stream; every kernel is
launched by libdpb200.so.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

PRECISIONS = {"fp32": _lib.PREC_FP32, "mixed": _lib.PREC_MIXED}


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("deepmd_jax_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists")


def _ptr(t):
    """Raw device pointer for the C ABI; the ABI reads dense row-major
    arrays, so strided views are rejected instead of being misread."""
    if t is None:
        return ctypes.c_void_p(0)
    if not t.is_contiguous():
        raise ValueError("libdpb200 takes contiguous arrays; got strides %s for shape %s"
                         % (tuple(t.stride()), tuple(t.shape)))
    if not t.is_cuda:
        raise ValueError("libdpb200 takes CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class DeviceModel:
    """A se_a energy model resident on the current CUDA device.

    ``params`` / ``variables`` use the reference's model.pkl layout
    (deepmd_jax/train.py:288-304; variables['params'] as in
    deepmd_jax/dpmodel.py:50-81)."""

    def __init__(self, params, variables):
        _require_cuda()
        self.lib = _lib.load()
        p = params
        v = variables["params"]
        if p.get("use_mp", False) or p.get("atomic", False) or p.get("type", "energy") not in ("energy",):
            raise NotImplementedError("only se_a energy models (no message passing / atomic / dplr)")
        if not p.get("use_2nd", True):
            raise NotImplementedError("use_2nd=False models are not supported")
        compressed = bool(p.get("is_compressed", False))
        if compressed and "compress_var" not in variables:
            raise ValueError("params['is_compressed'] is set but variables has no 'compress_var'")
        self.params = p
        self.ntypes = int(p["ntypes"])
        self.rcut = float(p["rcut"])
        ew = list(p["embed_widths"])
        fw = list(p["fit_widths"])
        nt = self.ntypes
        keep = []

        def f32(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
            keep.append(a)
            return a.ctypes.data

        def f64(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
            keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

        ek, eb = [], []
        for k in range(nt * nt):
            net = v["embedding_net_%d" % k]
            for li in range(len(ew)):
                ek.append(f32(net["Dense_%d" % li]["kernel"]))
                eb.append(f32(net["Dense_%d" % li]["bias"]))
        fk, fb, fdt = [], [], []
        for t in range(nt):
            net = v["fitting_net_%d" % t]
            for li in range(len(fw) + 1):
                fk.append(f32(net["Dense_%d" % li]["kernel"]))
                fb.append(f32(net["Dense_%d" % li]["bias"]))
            for li in range(len(fw)):
                dt = net.get("dt%d" % li)
                fdt.append(f32(dt) if dt is not None else None)
        d = _lib.ModelDesc()
        d.ntypes = nt
        d.n_embed = len(ew)
        for i, w in enumerate(ew):
            d.embed_widths[i] = int(w)
        d.n_fit = len(fw)
        for i, w in enumerate(fw):
            d.fit_widths[i] = int(w)
        d.axis = int(p["axis"])
        d.rcut = float(p["rcut"])
        d.nnbrs = float(p["Nnbrs"])
        d.out_norm = float(p.get("out_norm", 1.0))
        d.sr_mean = f64(p["sr_mean"])
        d.sr_std = f64(p["sr_std"])
        d.ebias = f64(p["Ebias"])
        VP = ctypes.c_void_p
        self._arrs = [(VP * len(ek))(*ek), (VP * len(eb))(*eb), (VP * len(fk))(*fk), (VP * len(fb))(*fb),
                      (VP * len(fdt))(*[x if x is not None else None for x in fdt])]
        d.embed_kernel = ctypes.cast(self._arrs[0], ctypes.POINTER(VP))
        d.embed_bias = ctypes.cast(self._arrs[1], ctypes.POINTER(VP))
        d.tbias = f32(v["Tbias"])
        d.fit_kernel = ctypes.cast(self._arrs[2], ctypes.POINTER(VP))
        d.fit_bias = ctypes.cast(self._arrs[3], ctypes.POINTER(VP))
        d.fit_dt = ctypes.cast(self._arrs[4], ctypes.POINTER(VP))
        if compressed:
            # piecewise quintic tables of compress_model (deepmd_jax/utils.py:250-297)
            cv = variables["compress_var"]
            coeff, lo, hi = [], [], []
            for k in range(nt * nt):
                e = cv["embedding_net_%d" % k]
                pc = np.asarray(e["poly_coeff"])
                if pc.ndim != 3 or pc.shape[1] != 6 or pc.shape[2] != int(ew[-1]):
                    raise ValueError("poly_coeff of embedding_net_%d has shape %s" % (k, pc.shape))
                coeff.append(f32(pc))
                lo.append(float(np.asarray(e["srmin"])))
                hi.append(float(np.asarray(e["srmax"])))
            ngrids = {int(np.asarray(cv["embedding_net_%d" % k]["poly_coeff"]).shape[0]) for k in range(nt * nt)}
            if len(ngrids) != 1:
                raise NotImplementedError("embedding tables with different grid counts")
            d.n_grids = ngrids.pop()
            self._arrs.append((VP * len(coeff))(*coeff))
            d.cmp_coeff = ctypes.cast(self._arrs[-1], ctypes.POINTER(VP))
            d.cmp_srmin = f64(lo)
            d.cmp_srmax = f64(hi)
        self.compressed = compressed
        h = ctypes.c_void_p()
        _lib.check(self.lib.dpb_model_create(ctypes.byref(d), ctypes.byref(h)), "dpb_model_create")
        self.handle = h
        self._ws = None
        del keep

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and self.handle.value:
                self.lib.dpb_model_destroy(self.handle)
        except Exception:
            pass

    # -- workspace -------------------------------------------------------------
    def eval_workspace(self, natoms, nframes):
        n = ctypes.c_size_t()
        _lib.check(self.lib.dpb_eval_workspace_bytes(self.handle, natoms, nframes, ctypes.byref(n)),
                   "dpb_eval_workspace_bytes")
        if self._ws is None or self._ws.numel() < n.value:
            self._ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
        return self._ws

    # -- evaluation ------------------------------------------------------------
    def evaluate(self, pos, box, nbrs, type_count, sel, perm=None, precision="fp32", atom_energy=False,
                 out=None, status=None, workspace=None):
        """pos (F,N,3) f32 cuda, box (F,3) f32 cuda, nbrs (F,N,S) int32 cuda.
        Returns dict(energy (F,) f64, force (F,N,3) f32, virial (F,9) f64,
        atom_energy (F,N) f32 or None, status (1,) int32)."""
        F, N = pos.shape[0], pos.shape[1]
        dev = pos.device
        if out is None:
            out = dict(energy=torch.empty(F, dtype=torch.float64, device=dev),
                       force=torch.empty((F, N, 3), dtype=torch.float32, device=dev),
                       virial=torch.empty((F, 9), dtype=torch.float64, device=dev),
                       atom_energy=torch.empty((F, N), dtype=torch.float32, device=dev) if atom_energy else None)
        if status is None:
            status = torch.zeros(1, dtype=torch.int32, device=dev)
        ws = workspace if workspace is not None else self.eval_workspace(N, F)
        rc = self.lib.dpb_eval(self.handle, PRECISIONS[precision], _ptr(pos), _ptr(perm), N, F,
                               _lib.int_array(type_count), _ptr(box), _ptr(nbrs), _lib.int_array(sel),
                               _ptr(out["energy"]), _ptr(out.get("atom_energy")), _ptr(out["force"]),
                               _ptr(out["virial"]), _ptr(status), _ptr(ws), ws.numel(), _stream())
        _lib.check(rc, "dpb_eval")
        out["status"] = status
        return out

    def descriptors(self, pos, box, nbrs, type_count, sel, perm=None, precision="fp32"):
        """The descriptor stage alone: T (F*N, 10, W) / Nnbrs without Tbias
        (the reference's T_NselXW, deepmd_jax/dpmodel.py:50-51) and G (F*N,
        A*W), atoms in type-sorted order, float32 on the device."""
        F, N = pos.shape[0], pos.shape[1]
        W, A = int(self.params["embed_widths"][-1]), int(self.params["axis"])
        dev = pos.device
        T = torch.empty((F * N, 10, W), dtype=torch.float32, device=dev)
        G = torch.empty((F * N, A * W), dtype=torch.float32, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        ws = self.eval_workspace(N, F)
        rc = self.lib.dpb_eval_descriptors(self.handle, PRECISIONS[precision], _ptr(pos), _ptr(perm), N, F,
                                           _lib.int_array(type_count), _ptr(box), _ptr(nbrs), _lib.int_array(sel),
                                           _ptr(T), _ptr(G), _ptr(err), _ptr(ws), ws.numel(), _stream())
        _lib.check(rc, "dpb_eval_descriptors")
        return T, G


class NeighborBuilder:
    """Typed neighbour lists (reference nbrs_nm semantics) via dpb_nlist_build."""

    def __init__(self, natoms, nframes, type_count, sel, box, rcut_plus_skin, ref_box=None):
        _require_cuda()
        self.lib = _lib.load()
        self.N, self.F = int(natoms), int(nframes)
        self.type_count = [int(x) for x in type_count]
        self.sel = [int(x) for x in sel]
        self.box = [float(x) for x in box]
        self.ref_box = None if ref_box is None else [float(x) for x in ref_box]
        self.rc = float(rcut_plus_skin)
        n = ctypes.c_size_t()
        rb = self.ref_box if self.ref_box is not None else self.box
        _lib.check(self.lib.dpb_nlist_workspace_bytes(self.N, self.F, _lib.float3(rb), ctypes.c_float(self.rc * 0.999),
                                                      ctypes.byref(n)), "dpb_nlist_workspace_bytes")
        self.ws = torch.empty(max(n.value, 256), dtype=torch.uint8, device="cuda")

    def build(self, pos, perm=None, nbrs=None, ref_pos=None, counts=None, status=None):
        dev = pos.device
        S = sum(self.sel)
        if nbrs is None:
            nbrs = torch.empty((self.F, self.N, S), dtype=torch.int32, device=dev)
        if status is None:
            status = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = self.lib.dpb_nlist_build(_ptr(pos), _ptr(perm), self.N, self.F, len(self.type_count),
                                      _lib.int_array(self.type_count), _lib.int_array(self.sel),
                                      _lib.float3(self.box),
                                      None if self.ref_box is None else _lib.float3(self.ref_box),
                                      ctypes.c_float(self.rc), _ptr(nbrs), _ptr(ref_pos), _ptr(counts),
                                      _ptr(status), _ptr(self.ws), self.ws.numel(), _stream())
        _lib.check(rc, "dpb_nlist_build")
        return nbrs, status


def sort_by_type(type_idx, ntypes):
    type_idx = np.asarray(type_idx)
    perm = np.argsort(type_idx, kind="stable")
    count = np.bincount(type_idx, minlength=ntypes)
    return perm, count


def _pad8(n):
    return (int(n) + 7) // 8 * 8


class PackedBatch:
    """Host layout of many request frames packed into one evaluation
    (dpb_eval_packed / dpb_nlist_pack).

    ``items`` is a list of (type_idx (N,), nframes, box (3,)); the frames of
    one item share the atom order, the type counts and the box.  Segment
    s numbers the frames item after item.  Packed type block t holds, item
    after item and frame after frame, each frame's type-t atoms padded to a
    multiple of 8; the slots (rows of the position / force buffers) are the
    items' frames in their own atom order, then one slot per padding atom."""

    def __init__(self, items, ntypes):
        self.ntypes = ntypes
        self.items = []
        counts = []
        for type_idx, nframes, box in items:
            perm, cnt = sort_by_type(np.asarray(type_idx), ntypes)
            counts.append((perm, cnt, int(nframes), np.asarray(box, np.float32).reshape(3)))
        pad = np.array([[_pad8(c) for c in cnt] for _, cnt, _, _ in counts], dtype=np.int64).reshape(-1, ntypes)
        nfr = np.array([nf for _, _, nf, _ in counts], dtype=np.int64)
        self.type_count = [int((pad[:, t] * nfr).sum()) for t in range(ntypes)]
        self.natoms = int(sum(self.type_count))
        offs = np.concatenate([[0], np.cumsum(self.type_count)]).astype(np.int64)
        perm_p = np.empty(self.natoms, dtype=np.int64)
        seg_p = np.empty(self.natoms, dtype=np.int64)
        self.nreal = int(sum(len(p) * nf for p, _, nf, _ in counts))
        dummy_next = self.nreal
        base = np.zeros(ntypes, dtype=np.int64)
        u0, s0 = 0, 0
        boxes = []
        for (perm, cnt, nf, box), pd in zip(counts, pad):
            N = len(perm)
            soffs = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
            it = {"natoms": N, "nframes": nf, "slot0": u0, "seg0": s0, "perm": perm, "type_count": cnt,
                  "row0": [], "base0": [], "stride": [], "box": box}
            for t in range(ntypes):
                p, n = int(pd[t]), int(cnt[t])
                it["row0"].append(int(offs[t] + base[t]))
                it["base0"].append(int(base[t]))
                it["stride"].append(p)
                rows = offs[t] + base[t] + np.arange(nf)[:, None] * p + np.arange(p)[None, :]   # (nf, p)
                real = u0 + np.arange(nf)[:, None] * N + perm[soffs[t]:soffs[t + 1]][None, :]   # (nf, n)
                nd = nf * (p - n)
                dummies = np.arange(dummy_next, dummy_next + nd).reshape(nf, p - n)
                dummy_next += nd
                perm_p[rows] = np.concatenate([real, dummies], axis=1)
                s = s0 + np.arange(nf)[:, None]
                seg_p[rows] = np.concatenate([np.broadcast_to(s, (nf, n)), np.broadcast_to(-(s + 1), (nf, p - n))],
                                             axis=1)
                base[t] += nf * p
            boxes += [box] * nf
            self.items.append(it)
            u0 += nf * N
            s0 += nf
        self.nseg = s0
        self.perm = perm_p.astype(np.int32)
        self.seg = seg_p.astype(np.int32)
        self.boxes = np.asarray(boxes, np.float32).reshape(-1, 3)


def evaluate_packed(dm, batch, slot_pos, sel, rcut, precision="fp32", atom_energy=False, host_stage=None):
    """One packed evaluation of every frame of ``batch`` (a PackedBatch).

    slot_pos: (batch.natoms, 3) float32 CUDA, the frames' positions at their
    slots (padding slots any finite value).  host_stage: optional pinned
    int32 host tensor that stages the batch's index arrays (the caller keeps
    it untouched until this batch completes); without it one is allocated.
    Returns energy (nseg,) f64, force (natoms, 3) f32 at the slots, virial
    (nseg, 9) f64, status."""
    lib = dm.lib
    dev = slot_pos.device
    Np, S = batch.natoms, int(sum(sel))
    nbrs = torch.full((Np, S), Np, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    # every host array of the batch (the items' type orders, the packed order,
    # the segments, the boxes as float bits) in one pinned buffer and one
    # asynchronous copy, so the host does not wait on the stream per item
    parts = [it["perm"].astype(np.int32) for it in batch.items] + [batch.perm, batch.seg,
                                                                    batch.boxes.reshape(-1).view(np.int32)]
    offs = np.concatenate([[0], np.cumsum([len(x) for x in parts])])
    if host_stage is not None and host_stage.numel() >= int(offs[-1]):
        host = host_stage[:int(offs[-1])]
    else:
        host = torch.empty(int(offs[-1]), dtype=torch.int32, pin_memory=True)
    hv = host.numpy()
    for x, o in zip(parts, offs[:-1]):
        hv[o:o + len(x)] = x
    dbuf = host.to(dev, non_blocking=True)
    views = [dbuf[offs[i]:offs[i + 1]] for i in range(len(parts))]
    for it, perm in zip(batch.items, views):
        N, nf = it["natoms"], it["nframes"]
        pos = slot_pos[it["slot0"]:it["slot0"] + nf * N].view(nf, N, 3)
        nb, _ = NeighborBuilder(N, nf, it["type_count"], sel, it["box"], rcut).build(pos, perm=perm, status=status)
        _lib.check(lib.dpb_nlist_pack(_ptr(nb), N, nf, batch.ntypes, _lib.int_array(it["type_count"]),
                                      _lib.int_array(sel), _lib.int_array(it["row0"]), _lib.int_array(it["base0"]),
                                      _lib.int_array(it["stride"]), Np, _ptr(nbrs), _stream()), "dpb_nlist_pack")
    n = ctypes.c_size_t()
    _lib.check(lib.dpb_eval_packed_workspace_bytes(dm.handle, Np, batch.nseg, ctypes.byref(n)),
               "dpb_eval_packed_workspace_bytes")
    ws = torch.empty(n.value, dtype=torch.uint8, device=dev)
    perm, seg = views[-3], views[-2]
    box = views[-1].view(torch.float32)
    out = dict(energy=torch.empty(batch.nseg, dtype=torch.float64, device=dev),
               force=torch.empty((Np, 3), dtype=torch.float32, device=dev),
               virial=torch.empty((batch.nseg, 9), dtype=torch.float64, device=dev),
               atom_energy=torch.empty(Np, dtype=torch.float32, device=dev) if atom_energy else None)
    rc = lib.dpb_eval_packed(dm.handle, PRECISIONS[precision], _ptr(slot_pos), _ptr(perm), Np,
                             _lib.int_array(batch.type_count), _ptr(seg), batch.nseg, _ptr(box), _ptr(nbrs),
                             _lib.int_array(sel), _ptr(out["energy"]), _ptr(out["atom_energy"]), _ptr(out["force"]),
                             _ptr(out["virial"]), _ptr(status), _ptr(ws), ws.numel(), _stream())
    _lib.check(rc, "dpb_eval_packed")
    out["status"] = status
    out["nbrs"] = nbrs
    return out
