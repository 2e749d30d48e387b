"""Minimal torch-backed stand-in for the parts of jax / flax.linen that the
reference's model source (deepmd_jax/utils.py, deepmd_jax/dpmodel.py,
deepmd_jax/data.py:347-364, deepmd_jax/pimd.py) touches on the energy path.

Test infrastructure only: make_golden.py installs these modules into
sys.modules, imports the UNMODIFIED reference files from the reference
checkout and runs them in float64 to produce golden vectors.  Nothing in the
product imports this file.

Semantics reproduced from jax where torch differs:
  * integer-array gathers clamp out-of-range indices (jax's default
    "clip"/"fill-free" gather), negative indices wrap;
  * ``x.transpose(*perm)`` permutes like numpy; ``astype``;
  * mixed int/float ``@`` promotes to float;
  * flax.linen submodule auto-naming ``ClassName_{k}`` per parent scope,
    ``self.param`` / ``self.variable`` lookups by scope path,
    ``nn.Dense`` = x @ kernel + bias.
"""
from __future__ import annotations

import dataclasses
import sys
import types

import numpy as np
import torch

DT = torch.float64


class JArray(torch.Tensor):
    """torch tensor with numpy/jax-style methods the reference uses."""

    def transpose(self, *axes):
        if len(axes) == 1 and isinstance(axes[0], (tuple, list)):
            axes = tuple(axes[0])
        if len(axes) == 0:
            axes = tuple(reversed(range(self.dim())))
        return self.permute(*axes)

    @property
    def T(self):
        return self.permute(*reversed(range(self.dim())))

    def astype(self, dt):
        return self.to(_dtype(dt))

    def any(self, axis=None, *a, **k):
        if axis is None:
            return torch.Tensor.any(self)
        if isinstance(axis, tuple):
            out = self
            for d in sorted([d % self.dim() for d in axis], reverse=True):
                out = torch.Tensor.any(out, dim=d)
            return out
        return torch.Tensor.any(self, dim=axis)

    # jax arrays are immutable: augmented assignment rebinds, never mutates
    def __iadd__(self, other):
        return self + other

    def __isub__(self, other):
        return self - other

    def __imul__(self, other):
        return self * other

    def __itruediv__(self, other):
        return self / other

    def max(self, axis=None, *a, **k):
        if axis is None:
            return torch.Tensor.max(self)
        return torch.Tensor.max(self, dim=axis).values

    def min(self, axis=None, *a, **k):
        if axis is None:
            return torch.Tensor.min(self)
        return torch.Tensor.min(self, dim=axis).values

    def __getitem__(self, idx):
        return torch.Tensor.__getitem__(self, _clamp_index(self, idx))

    def __matmul__(self, other):
        a, b = _promote(self, other)
        return torch.matmul(a, b)

    def __rmatmul__(self, other):
        a, b = _promote(other, self)
        return torch.matmul(a, b)

    @property
    def nbytes(self):
        return self.element_size() * self.numel()


def _promote(a, b):
    a = a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a))
    b = b if torch.is_tensor(b) else torch.as_tensor(np.asarray(b))
    if a.dtype != b.dtype:
        dt = torch.promote_types(a.dtype, b.dtype)
        if not dt.is_floating_point and (a.is_floating_point() or b.is_floating_point()):
            dt = DT
        a, b = a.to(dt), b.to(dt)
    return a, b


def _clamp_index(t, idx):
    single = not isinstance(idx, tuple)
    items = (idx,) if single else idx
    out, dim = [], 0
    for it in items:
        if it is None:
            out.append(it)
            continue
        if it is Ellipsis:
            # account for dims consumed after the ellipsis
            rest = sum(1 for x in items[items.index(Ellipsis) + 1:] if x is not None)
            dim = t.dim() - rest
            out.append(it)
            continue
        if isinstance(it, np.ndarray):
            it = torch.as_tensor(it)
        if torch.is_tensor(it) and not it.dtype.is_floating_point and it.dtype != torch.bool:
            n = t.shape[dim]
            it = torch.where(it < 0, it + n, it).clamp(0, max(n - 1, 0)).to(torch.int64)
            out.append(it.as_subclass(torch.Tensor))
            dim += 1
            continue
        out.append(it)
        dim += 1
    return out[0] if single else tuple(out)


def _dtype(dt):
    if dt is None:
        return None
    if isinstance(dt, torch.dtype):
        return dt
    if dt is bool:
        return torch.bool
    if dt is int:
        return torch.int64
    if dt is float:
        return DT
    return {np.dtype("float32"): torch.float32, np.dtype("float64"): torch.float64,
            np.dtype("int32"): torch.int32, np.dtype("int64"): torch.int64,
            np.dtype("bool"): torch.bool}[np.dtype(dt)]


def J(x, dtype=None):
    if torch.is_tensor(x):
        t = x if dtype is None else x.to(_dtype(dtype))
    else:
        a = np.asarray(x)
        if a.dtype == np.float32:
            a = a.astype(np.float64)
        t = torch.as_tensor(a)
        if dtype is not None:
            t = t.to(_dtype(dtype))
    return t.as_subclass(JArray)


# ----------------------------------------------------------------------------- jax.numpy
jnp = types.ModuleType("jax.numpy")
jnp.array = J
jnp.asarray = J
jnp.float32 = torch.float64   # run the reference graph in float64
jnp.float64 = torch.float64
jnp.int32 = torch.int32
jnp.ndarray = torch.Tensor
jnp.pi = np.pi
jnp.ones = lambda shape, dtype=None: torch.ones(shape, dtype=_dtype(dtype) or DT).as_subclass(JArray)
jnp.zeros = lambda shape, dtype=None: torch.zeros(shape, dtype=_dtype(dtype) or DT).as_subclass(JArray)
jnp.ones_like = lambda x, dtype=None: torch.ones_like(J(x), dtype=_dtype(dtype)).as_subclass(JArray)
jnp.zeros_like = lambda x, dtype=None: torch.zeros_like(J(x), dtype=_dtype(dtype)).as_subclass(JArray)
jnp.eye = lambda n, dtype=None: torch.eye(n, dtype=_dtype(dtype) or DT).as_subclass(JArray)


def _concatenate(arrs, axis=0):
    arrs = [J(a) for a in arrs]
    a0, rest = arrs[0], arrs[1:]
    dt = a0.dtype
    for a in rest:
        dt = torch.promote_types(dt, a.dtype)
    return torch.cat([a.to(dt) for a in arrs], dim=axis).as_subclass(JArray)


jnp.concatenate = _concatenate
jnp.stack = lambda arrs, axis=0: torch.stack([J(a) for a in arrs], dim=axis).as_subclass(JArray)
jnp.split = lambda a, idx, axis=0: [t.as_subclass(JArray) for t in torch.tensor_split(J(a), [int(i) for i in np.asarray(idx).reshape(-1)], dim=axis)]
jnp.repeat = lambda a, r, axis=None: torch.repeat_interleave(J(a), int(r), dim=axis).as_subclass(JArray)
jnp.roll = lambda a, shift, axis=None: torch.roll(J(a), shifts=shift, dims=axis).as_subclass(JArray)
jnp.where = lambda c, a, b: torch.where(J(c).bool(), *_promote(J(a), J(b))).as_subclass(JArray)
jnp.abs = lambda a: torch.abs(J(a)).as_subclass(JArray)
jnp.exp = lambda a: torch.exp(J(a)).as_subclass(JArray)
jnp.sqrt = lambda a: torch.sqrt(J(a)).as_subclass(JArray)
jnp.cos = lambda a: torch.cos(J(a)).as_subclass(JArray)
jnp.sin = lambda a: torch.sin(J(a)).as_subclass(JArray)
jnp.round = lambda a: torch.round(J(a)).as_subclass(JArray)
jnp.maximum = lambda a, b: torch.maximum(*_promote(J(a), J(b))).as_subclass(JArray)
jnp.prod = lambda a, axis=None: (torch.prod(J(a)) if axis is None else torch.prod(J(a), dim=axis)).as_subclass(JArray)
jnp.sum = lambda a, axis=None: (torch.sum(J(a)) if axis is None else torch.sum(J(a), dim=axis)).as_subclass(JArray)
jnp.tensordot = lambda a, b, axes: torch.tensordot(*_promote(J(a), J(b)), dims=axes).as_subclass(JArray)
jnp.take_along_axis = lambda a, idx, axis: torch.take_along_dim(J(a), J(idx).long(), dim=axis).as_subclass(JArray)
jnp.argpartition = lambda a, k, axis=-1: torch.argsort(J(a), dim=axis, stable=True).as_subclass(JArray)


def _diag(a):
    a = J(a)
    return torch.diag(a).as_subclass(JArray)


jnp.diag = _diag
jnp.linalg = types.SimpleNamespace(
    norm=lambda a, axis=None: torch.linalg.norm(J(a), dim=axis).as_subclass(JArray),
    inv=lambda a: torch.linalg.inv(J(a)).as_subclass(JArray),
    det=lambda a: torch.linalg.det(J(a)).as_subclass(JArray),
)

# ----------------------------------------------------------------------------- jax
jax = types.ModuleType("jax")
jax.numpy = jnp
jax.jit = lambda f=None, **kw: (f if f is not None else (lambda g: g))
jax.device_count = lambda: 1
jax.devices = lambda: ["cpu"]


def _vmap(f, in_axes=0, *a, **k):
    def g(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = next(J(x).shape[ax] for x, ax in zip(args, axes) if ax is not None)
        outs = [f(*[(J(x)[i] if ax is not None else x) for x, ax in zip(args, axes)]) for i in range(n)]
        if isinstance(outs[0], (tuple, list)):
            return type(outs[0])(jnp.stack([o[t] for o in outs]) for t in range(len(outs[0])))
        return jnp.stack(outs)
    return g


jax.vmap = _vmap
lax = types.ModuleType("jax.lax")
lax.with_sharding_constraint = lambda x, spec: x
lax.stop_gradient = lambda x: J(x).detach().as_subclass(JArray)
jax.lax = lax
jax.jacfwd = None
jax.value_and_grad = None
jax.grad = None
sharding = types.ModuleType("jax.sharding")
sharding.PartitionSpec = lambda *a: None
jax.sharding = sharding

# noise source for jax.random.normal, set by the golden generator
_NOISE = {"fn": None}
jrandom = types.ModuleType("jax.random")
jrandom.split = lambda key, n=2: (key, key)
jrandom.PRNGKey = lambda s: s
jrandom.normal = lambda key, shape=(), dtype=None: J(_NOISE["fn"](tuple(shape)))
jax.random = jrandom

_inits = types.SimpleNamespace(
    he_normal=lambda *a, **k: None,
    variance_scaling=lambda *a, **k: None,
    truncated_normal=lambda *a, **k: None,
    normal=lambda *a, **k: None,
    ones_init=lambda *a, **k: None,
    zeros_init=lambda *a, **k: None,
)
jnn = types.ModuleType("jax.nn")
jnn.initializers = _inits
jax.nn = jnn
jax.config = types.SimpleNamespace(update=lambda *a: None, read=lambda *a: False)

# ----------------------------------------------------------------------------- flax.linen


class _Scope:
    def __init__(self, variables, path=()):
        self.variables = variables
        self.path = path

    def lookup(self, collection, name):
        d = self.variables[collection]
        for p in self.path:
            d = d[p]
        return d[name]


_CTX = []


class Module:
    """flax.linen.Module stand-in: dataclass fields, compact submodules,
    param/variable lookup by scope path, auto names ClassName_k per parent."""

    def __init_subclass__(cls, **kw):
        super().__init_subclass__(**kw)
        if "__annotations__" in cls.__dict__:
            dataclasses.dataclass(cls, eq=False)
        if "__call__" in cls.__dict__:
            cls.__call__ = _auto_bind(cls.__dict__["__call__"])

    def _bind(self, scope):
        self._scope = scope
        self._counter = {}

    def apply(self, variables, *args, method=None, **kwargs):
        self._bind(_Scope(variables))
        if method is None:
            return self.__call__(*args, **kwargs)
        return method(self, *args, **kwargs)

    def param(self, name, init_fn, shape=None, *a):
        return J(self._scope.lookup("params", name))

    def variable(self, collection, name, *a):
        return types.SimpleNamespace(value=J(self._scope.lookup(collection, name)))

    def _child(self, child):
        prefix = type(child).__name__
        k = self._counter.get(prefix, 0)
        self._counter[prefix] = k + 1
        child._bind(_Scope(self._scope.variables, self._scope.path + ("%s_%d" % (prefix, k),)))
        return child


def _auto_bind(orig_call):
    def call(self, *args, **kwargs):
        if not hasattr(self, "_scope"):
            _CTX[-1]._child(self)
        _CTX.append(self)
        try:
            return orig_call(self, *args, **kwargs)
        finally:
            _CTX.pop()
    return call


def compact(fn):
    return fn


class Dense(Module):
    features: int
    kernel_init: object = None
    bias_init: object = None
    use_bias: bool = True

    def __call__(self, x):
        y = J(x) @ self.param("kernel", None)
        if self.use_bias:
            y = y + self.param("bias", None)
        return y


linen = types.ModuleType("flax.linen")
linen.Module = Module
linen.compact = compact
linen.Dense = Dense
linen.tanh = lambda x: torch.tanh(J(x)).as_subclass(JArray)
linen.initializers = _inits
linen.FrozenDict = dict
flax = types.ModuleType("flax")
flax.linen = linen


def install():
    """Register the stand-ins in sys.modules (plus empty stubs for modules the
    reference imports at top level but does not use on the energy path).
    torch's default dtype becomes float64 so that int-array x 0-d-float
    products promote to float64 as they do in jax with x64 enabled."""
    torch.set_default_dtype(torch.float64)
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.lax"] = lax
    sys.modules["jax.sharding"] = sharding
    sys.modules["jax.random"] = jrandom
    sys.modules["jax.nn"] = jnn
    sys.modules["flax"] = flax
    sys.modules["flax.linen"] = linen
    ase = types.ModuleType("ase")
    ase_io = types.ModuleType("ase.io")
    ase_io.read = None
    ase.io = ase_io
    sys.modules.setdefault("ase", ase)
    sys.modules.setdefault("ase.io", ase_io)
    jax_md = types.ModuleType("jax_md")
    jax_md.dataclasses = types.SimpleNamespace(dataclass=dataclasses.dataclass,
                                               static_field=lambda: dataclasses.field(default=None))
    jax_md.simulate = types.SimpleNamespace()
    sys.modules.setdefault("jax_md", jax_md)


def load_reference(ref_root):
    """Import deepmd_jax.{utils,dpmodel,data,pimd} from the reference checkout
    without running its package __init__ (which configures real jax)."""
    import importlib
    install()
    pkg = types.ModuleType("deepmd_jax")
    pkg.__path__ = [str(ref_root) + "/deepmd_jax"]
    sys.modules["deepmd_jax"] = pkg
    mods = {}
    for name in ("utils", "dpmodel", "data", "pimd"):
        mods[name] = importlib.import_module("deepmd_jax." + name)
    return mods
