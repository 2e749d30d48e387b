"""ctypes binding of libdpb200.so (the C ABI declared in include/dpb200.h).

The shared library is built in-tree (deepmd_jax_b200/lib/libdpb200.so) by
``deepmd-jax_b200/csrc/Makefile``.  There is no fallback: if the library or
a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libdpb200.so")

DPB_OK = 0
STATUS_BITS = {1: "box shrank past the skin", 2: "neighbour list overflow", 4: "overflow in previous chunk",
               8: "lattice overflow", 16: "NaN/Inf encountered"}
ERRORS = {256: "DPB_ERR_INVALID_ARG", 257: "DPB_ERR_CUDA", 258: "DPB_ERR_UNSUPPORTED",
          259: "DPB_ERR_WORKSPACE", 260: "DPB_ERR_NO_DEVICE", 261: "DPB_ERR_SCRATCH_LIMIT"}
PREC_FP32 = 0
PREC_MIXED = 1
NBR_INDEX_MASK = 0x00FFFFFF

EXPORTED = ["dpb_model_create", "dpb_model_destroy", "dpb_nlist_workspace_bytes", "dpb_nlist_build",
            "dpb_eval_workspace_bytes", "dpb_eval", "dpb_eval_noalloc", "dpb_eval_packed_workspace_bytes",
            "dpb_eval_packed", "dpb_nlist_pack", "dpb_kernel_launch_count", "dpb_version"]


class DPBError(RuntimeError):
    def __init__(self, code, what=""):
        super().__init__("%s failed: %s (%d)" % (what, ERRORS.get(code, "unknown"), code))
        self.code = code


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("ntypes", ctypes.c_int),
        ("n_embed", ctypes.c_int),
        ("embed_widths", ctypes.c_int * 4),
        ("n_fit", ctypes.c_int),
        ("fit_widths", ctypes.c_int * 4),
        ("axis", ctypes.c_int),
        ("rcut", ctypes.c_double),
        ("nnbrs", ctypes.c_double),
        ("out_norm", ctypes.c_double),
        ("sr_mean", ctypes.POINTER(ctypes.c_double)),
        ("sr_std", ctypes.POINTER(ctypes.c_double)),
        ("ebias", ctypes.POINTER(ctypes.c_double)),
        ("embed_kernel", ctypes.POINTER(ctypes.c_void_p)),
        ("embed_bias", ctypes.POINTER(ctypes.c_void_p)),
        ("tbias", ctypes.c_void_p),
        ("fit_kernel", ctypes.POINTER(ctypes.c_void_p)),
        ("fit_bias", ctypes.POINTER(ctypes.c_void_p)),
        ("fit_dt", ctypes.POINTER(ctypes.c_void_p)),
        ("n_grids", ctypes.c_int),
        ("cmp_coeff", ctypes.POINTER(ctypes.c_void_p)),
        ("cmp_srmin", ctypes.POINTER(ctypes.c_double)),
        ("cmp_srmax", ctypes.POINTER(ctypes.c_double)),
    ]


_lib = None


def load():
    """Load libdpb200.so once and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("libdpb200.so not built: run `make -C deepmd-jax_b200/csrc` (expected at %s)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32p, f32p, f64p = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p
    c_int_p = ctypes.POINTER(ctypes.c_int)
    f3 = ctypes.POINTER(ctypes.c_float)
    lib.dpb_model_create.argtypes = [ctypes.POINTER(ModelDesc), ctypes.POINTER(ctypes.c_void_p)]
    lib.dpb_model_create.restype = ctypes.c_int
    lib.dpb_model_destroy.argtypes = [vp]
    lib.dpb_model_destroy.restype = ctypes.c_int
    lib.dpb_nlist_workspace_bytes.argtypes = [ctypes.c_int, ctypes.c_int, f3, ctypes.c_float,
                                              ctypes.POINTER(ctypes.c_size_t)]
    lib.dpb_nlist_workspace_bytes.restype = ctypes.c_int
    lib.dpb_nlist_build.argtypes = [f32p, i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p, c_int_p,
                                    f3, f3, ctypes.c_float, i32p, f32p, i32p, vp, vp, ctypes.c_size_t, vp]
    lib.dpb_nlist_build.restype = ctypes.c_int
    lib.dpb_eval_workspace_bytes.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    lib.dpb_eval_workspace_bytes.restype = ctypes.c_int
    lib.dpb_eval_descriptors.argtypes = [vp, ctypes.c_int, f32p, i32p, ctypes.c_int, ctypes.c_int, c_int_p, f32p,
                                         i32p, c_int_p, vp, vp, vp, vp, ctypes.c_size_t, vp]
    lib.dpb_eval_descriptors.restype = ctypes.c_int
    lib.dpb_eval.argtypes = [vp, ctypes.c_int, f32p, i32p, ctypes.c_int, ctypes.c_int, c_int_p, f32p, i32p,
                             c_int_p, f64p, f32p, f32p, f64p, vp, vp, ctypes.c_size_t, vp]
    lib.dpb_eval.restype = ctypes.c_int
    lib.dpb_eval_noalloc.argtypes = [vp, ctypes.c_int, f32p, i32p, ctypes.c_int, ctypes.c_int, c_int_p, f32p, i32p,
                                     c_int_p, f64p, f32p, f32p, f64p, vp, vp]
    lib.dpb_eval_noalloc.restype = ctypes.c_int
    lib.dpb_eval_packed_workspace_bytes.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    lib.dpb_eval_packed_workspace_bytes.restype = ctypes.c_int
    lib.dpb_eval_packed.argtypes = [vp, ctypes.c_int, f32p, i32p, ctypes.c_int, c_int_p, i32p, ctypes.c_int, f32p,
                                    i32p, c_int_p, f64p, f32p, f32p, f64p, vp, vp, ctypes.c_size_t, vp]
    lib.dpb_eval_packed.restype = ctypes.c_int
    lib.dpb_nlist_pack.argtypes = [i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p, c_int_p, c_int_p, c_int_p,
                                   c_int_p, ctypes.c_int, i32p, vp]
    lib.dpb_nlist_pack.restype = ctypes.c_int
    lib.dpb_kernel_launch_count.argtypes = []
    lib.dpb_kernel_launch_count.restype = ctypes.c_uint64
    lib.dpb_version.argtypes = []
    lib.dpb_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(rc, what):
    if rc != DPB_OK:
        raise DPBError(rc, what)


def int_array(vals):
    arr = (ctypes.c_int * len(vals))(*[int(v) for v in vals])
    return arr


def float3(vals):
    return (ctypes.c_float * 3)(*[float(v) for v in vals])
