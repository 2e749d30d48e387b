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
