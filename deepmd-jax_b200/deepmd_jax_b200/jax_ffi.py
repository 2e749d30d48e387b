"""jax.ffi custom calls over libdpb200 (the shim built from
csrc/jax_ffi/dpb_jax_ffi.cc where jaxlib's FFI headers exist).

``register()`` loads lib/libdpb_jax_ffi.so and registers its two handlers
for the CUDA platform; ``energy_and_force`` and ``nlist_build`` are the
jax-side calls a deepmd-jax maintainer puts in place of
``DPModel.energy_and_force`` (deepmd_jax/dpmodel.py:106-108, used by the force
function of md.py:292) and of ``typed_neighbor_list(...).allocate/update``
(md_utils.py:376-429).  jax is imported lazily: without it these raise
ImportError, and nothing else in the package needs it.
"""
from __future__ import annotations

import ctypes
import os

_REGISTERED = None


def library_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libdpb_jax_ffi.so")


def register():
    """Register dpb_eval / dpb_nlist_build as jax.ffi targets (once)."""
    global _REGISTERED
    if _REGISTERED is not None:
        return _REGISTERED
    import jax
    from . import _lib
    _lib.load()  # libdpb200 first, so the shim's dependency resolves
    path = library_path()
    if not os.path.exists(path):
        raise ImportError("%s is not built (make -C deepmd-jax_b200/csrc/jax_ffi)" % path)
    shim = ctypes.CDLL(path)
    jax.ffi.register_ffi_target("dpb_eval", jax.ffi.pycapsule(shim.dpb_eval_ffi), platform="CUDA")
    jax.ffi.register_ffi_target("dpb_nlist_build", jax.ffi.pycapsule(shim.dpb_nlist_build_ffi), platform="CUDA")
    _REGISTERED = shim
    return shim


def energy_and_force(pos, perm, box, nbrs, model_handle, type_count, sel, workspace_bytes, precision=0):
    """(energy (F,) f64, force (F,N,3) f32, virial (F,9) f64, status (1,) u32)
    of frames pos (F,N,3) f32 with the typed list nbrs (F,N,sum(sel)) int32
    (the packed nbrs_nm: type-local ascending indices, pad N)."""
    import jax
    import jax.numpy as jnp
    register()
    F, N = pos.shape[:2]
    out = (jax.ShapeDtypeStruct((F,), jnp.float64), jax.ShapeDtypeStruct((F, N, 3), jnp.float32),
           jax.ShapeDtypeStruct((F, 9), jnp.float64), jax.ShapeDtypeStruct((1,), jnp.uint32),
           jax.ShapeDtypeStruct((int(workspace_bytes),), jnp.uint8))
    E, Fo, W, st, _ = jax.ffi.ffi_call("dpb_eval", out)(
        pos, perm, box, nbrs, model=int(model_handle), precision=int(precision),
        type_count=tuple(int(x) for x in type_count), sel=tuple(int(x) for x in sel))
    return E, Fo, W, st


def nlist_build(pos, perm, box, rcut_plus_skin, type_count, sel, workspace_bytes, ref_box=()):
    """(nbrs (F,N,sum(sel)) int32, reference positions (F,N,3), status (1,))
    of frames pos (F,N,3) f32 in a box given as three host floats."""
    import jax
    import jax.numpy as jnp
    import numpy as np
    register()
    F, N = pos.shape[:2]
    out = (jax.ShapeDtypeStruct((F, N, int(sum(sel))), jnp.int32), jax.ShapeDtypeStruct((F, N, 3), jnp.float32),
           jax.ShapeDtypeStruct((1,), jnp.uint32), jax.ShapeDtypeStruct((int(workspace_bytes),), jnp.uint8))
    nb, ref, st, _ = jax.ffi.ffi_call("dpb_nlist_build", out)(
        pos, perm, type_count=tuple(int(x) for x in type_count), sel=tuple(int(x) for x in sel),
        box=np.asarray(box, np.float32), ref_box=np.asarray(ref_box, np.float32),
        rcut_plus_skin=np.float32(rcut_plus_skin))
    return nb, ref, st
