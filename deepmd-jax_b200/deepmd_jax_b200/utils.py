"""Model I/O in the reference's model.pkl format.

The reference pickles ``{'model': DPModel(params), 'variables': pytree}``
(deepmd_jax/utils.py:225-237), where DPModel is a flax module and the leaves
are jax arrays.  Neither jax nor flax is needed here: ``load_model`` maps the
flax / jax classes the pickle names onto small stand-ins that keep the
``params`` dict and turn arrays into numpy, and ``save_model`` writes a pickle
that names the same classes, so the reference's loader can read it back where
jax and flax are installed.
"""
from __future__ import annotations

import io
import pickle
import sys
import types

import numpy as np


class DPModelStub:
    """Stand-in for deepmd_jax.dpmodel.DPModel: holds ``params``."""

    def __init__(self, params=None, **kw):
        self.params = params if params is not None else {}

    def __setstate__(self, state):
        if isinstance(state, tuple):  # (dict, slots)
            state = state[0] or {}
        self.__dict__.update(state)
        if "params" not in self.__dict__:
            self.params = {}

    def __reduce__(self):
        return (_dpmodel_class(), (), {"params": self.params, "parent": None, "name": None})


class _Opaque:
    """Flax module bookkeeping the pickle carries along (internal state
    dataclasses, the unspecified-parent sentinel): kept, never used."""

    def __init__(self, *a, **k):
        pass

    def __setstate__(self, state):
        if isinstance(state, tuple):  # (dict, slots)
            state = state[0] or {}
        if isinstance(state, dict):
            self.__dict__.update(state)


def _reconstruct_array(fun, args, arr_state, aval_state):
    """Stand-in for jax._src.array._reconstruct_array, the reducer jax.Array
    pickles through: (numpy's reconstructor, its args, the ndarray state, the
    abstract-value state).  Returns the numpy array."""
    a = fun(*args)
    a.__setstate__(arr_state)
    return np.asarray(a)


def _frozen_dict(*args, **kw):
    """flax.core.frozen_dict.FrozenDict pickles as FrozenDict(plain dict)."""
    return dict(*args, **kw)


def _enum_value(value):
    """Enum members (flax's SetupState) pickle as EnumClass(value)."""
    return value


def _none():
    return None


# Every global a reference model.pkl may name, and what it loads as.  The
# reference pickles {'model': DPModel (a flax Module), 'variables': pytree of
# jax.Array} (deepmd_jax/utils.py:225-228); a flax Module pickles as its class
# plus its instance dict (params, parent, name and flax's internal state), a
# jax.Array through jax._src.array._reconstruct_array over numpy's array
# reduction, a FrozenDict as FrozenDict(dict).  Anything else is refused.
_STANDINS = {
    ("deepmd_jax.dpmodel", "DPModel"): DPModelStub,
    ("jax._src.array", "_reconstruct_array"): _reconstruct_array,
    ("flax.core.frozen_dict", "FrozenDict"): _frozen_dict,
    ("flax.linen.module", "_ModuleInternalState"): _Opaque,
    ("flax.linen.module", "_Sentinel"): _Opaque,
    ("flax.linen.module", "SetupState"): _enum_value,
    ("flax.linen.module", "_get_unspecified_parent"): _none,
}
# numpy's own reducers (numpy 1.x names map to numpy 2.x's) and the plain
# containers pickle needs for older protocols.
_NUMPY = {
    ("numpy", "ndarray"): ("numpy", "ndarray"),
    ("numpy", "dtype"): ("numpy", "dtype"),
    ("numpy.core.multiarray", "_reconstruct"): ("numpy._core.multiarray", "_reconstruct"),
    ("numpy._core.multiarray", "_reconstruct"): ("numpy._core.multiarray", "_reconstruct"),
    ("numpy.core.multiarray", "scalar"): ("numpy._core.multiarray", "scalar"),
    ("numpy._core.multiarray", "scalar"): ("numpy._core.multiarray", "scalar"),
}
_PLAIN = {("builtins", n) for n in ("tuple", "list", "dict", "set", "frozenset", "complex", "bytearray", "object",
                                      "int", "float", "bool", "str", "bytes", "slice")}
_PLAIN |= {("collections", "OrderedDict"), ("copyreg", "_reconstructor"), ("_codecs", "encode")}


class _Unpickler(pickle.Unpickler):
    def find_class(self, module, name):
        key = (module, name)
        if key in _STANDINS:
            return _STANDINS[key]
        if key in _NUMPY:
            return super().find_class(*_NUMPY[key])
        if key in _PLAIN:
            return super().find_class(module, name)
        raise pickle.UnpicklingError("model.pkl refers to %s.%s, which is not allowed" % (module, name))


def _to_numpy_tree(x):
    if isinstance(x, dict):
        return {k: _to_numpy_tree(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return type(x)(_to_numpy_tree(v) for v in x)
    if hasattr(x, "__array__") and not isinstance(x, (str, bytes)):
        return np.asarray(x)
    return x


def load_model(path, replicate=True):
    """(model, variables) from a reference model.pkl; ``model.params`` is the
    parameter dict, ``variables`` a nested dict of numpy arrays."""
    with open(path, "rb") as f:
        m = _Unpickler(f).load()
    model = m["model"]
    if not isinstance(model, DPModelStub):
        model = DPModelStub(getattr(model, "params", {}))
    return model, _to_numpy_tree(m["variables"])


def _dpmodel_class():
    mod = sys.modules.get("deepmd_jax.dpmodel")
    if mod is None or not hasattr(mod, "DPModel"):
        mod = types.ModuleType("deepmd_jax.dpmodel")
        cls = type("DPModel", (DPModelStub,), {"__module__": "deepmd_jax.dpmodel"})
        mod.DPModel = cls
        pkg = sys.modules.get("deepmd_jax") or types.ModuleType("deepmd_jax")
        sys.modules.setdefault("deepmd_jax", pkg)
        sys.modules["deepmd_jax.dpmodel"] = mod
    return mod.DPModel


def save_model(path, model_or_params, variables):
    """Write ``{'model': DPModel(params), 'variables': variables}`` with the
    class path deepmd_jax.dpmodel.DPModel and numpy leaves."""
    params = getattr(model_or_params, "params", model_or_params)
    cls = _dpmodel_class()
    obj = cls.__new__(cls)
    obj.params = params
    with open(path, "wb") as f:
        pickle.dump({"model": obj, "variables": _to_numpy_tree(variables)}, f)


def sr(r, rcut):
    """1/r with the reference's smooth cutoff (deepmd_jax/utils.py:29-32), numpy."""
    r = np.asarray(r, dtype=float)
    t = r / rcut
    return ((r > 1e-14) & (t < 1)) / (r + 1e-15) * (1 - 3 * t ** 2 + 2 * t ** 3)


def _embedding_jet(layers, x):
    """Value, first and second derivative with respect to the scalar input
    of one embedding net (deepmd_jax/utils.py:100-125: tanh layers, each
    after the first plus its input repeated to the wider width, or averaged
    over groups where the width shrinks), float64, at the points x (n,)."""
    v = x[:, None].astype(np.float64)
    d1 = np.ones_like(v)
    d2 = np.zeros_like(v)
    for i, (Wk, b) in enumerate(layers):
        Wk = np.asarray(Wk, dtype=np.float64)
        z, z1, z2 = v @ Wk + np.asarray(b, dtype=np.float64), d1 @ Wk, d2 @ Wk
        t = np.tanh(z)
        g = 1.0 - t * t
        t1, t2 = g * z1, g * z2 - 2.0 * t * g * z1 * z1
        if i > 0:
            win, wout = Wk.shape
            if wout % win == 0:
                rep = lambda a: np.repeat(a, wout // win, axis=-1)  # noqa: E731
            else:
                rep = lambda a: a.reshape(a.shape[0], win // wout, wout).mean(1)  # noqa: E731
            t, t1, t2 = t + rep(v), t1 + rep(d1), t2 + rep(d2)
        v, d1, d2 = t, t1, t2
    return v, d1, d2


def _quintic_table(f0, f1, f2, h):
    """Coefficients (n, 6, W) in powers x0^5 .. x0^0 of the quintic on each
    interval [0, h] that takes the values, slopes and curvatures f0, f1, f2
    (n + 1, W) at both of its ends: the C2 piecewise quintic that the
    reference builds with scipy's BPoly.from_derivatives and converts to
    PPoly (deepmd_jax/utils.py:275-277)."""
    a0, a1, a2 = f0[:-1], f1[:-1], 0.5 * f2[:-1]
    # remaining conditions on a3 h^3 + a4 h^4 + a5 h^5 and its derivatives
    r0 = f0[1:] - (a0 + a1 * h + a2 * h * h)
    r1 = f1[1:] - (a1 + 2.0 * a2 * h)
    r2 = f2[1:] - 2.0 * a2
    # solution of [[h^3 h^4 h^5], [3h^2 4h^3 5h^4], [6h 12h^2 20h^3]] a = r
    a3 = (20.0 * r0 - 8.0 * h * r1 + h * h * r2) / (2.0 * h ** 3)
    a4 = (-30.0 * r0 + 14.0 * h * r1 - 2.0 * h * h * r2) / (2.0 * h ** 4)
    a5 = (12.0 * r0 - 6.0 * h * r1 + h * h * r2) / (2.0 * h ** 5)
    return np.stack([a5, a4, a3, a2, a1, a0], 1)


def compress_model(model, variables, Ngrids, rmin):
    """Tabulate every embedding net as a C2 piecewise quintic
    (deepmd_jax/utils.py:250-297): on Ngrids equal intervals of
    [srmin, srmax] = ([0, sr(rmin)] - sr_mean_i) / sr_std_i of the centre
    type i, the quintic matching the net's value and first two derivatives
    at both ends.  Sets model.params['is_compressed'] and
    variables['compress_var']['embedding_net_k'] = {srmin, srmax,
    poly_coeff (Ngrids, 6, W) float32}; returns (model, variables).
    Message-passing and atomic models are not supported."""
    params = model.params
    if params.get("use_mp") or params.get("atomic"):
        raise NotImplementedError("compress_model: message-passing and atomic models are not supported")
    params["is_compressed"] = True
    mean = np.asarray(params["sr_mean"], dtype=np.float64)
    std = np.asarray(params["sr_std"], dtype=np.float64)
    Y = len(mean)
    lo_hi = (np.array([0.0, float(sr(rmin, float(params["rcut"])))])[None, :] - mean[:, None]) / std[:, None]
    variables["compress_var"] = {}
    errs = [[], [], []]
    for k in range(Y * Y):
        name = "embedding_net_%d" % k
        net = variables["params"][name]
        nd = sum(1 for key in net if key.startswith("Dense_"))
        layers = [(net["Dense_%d" % i]["kernel"], net["Dense_%d" % i]["bias"]) for i in range(nd)]
        lo, hi = lo_hi[k // Y]
        r = np.linspace(lo, hi, Ngrids + 1)
        f0, f1, f2 = _embedding_jet(layers, r)
        coeff = _quintic_table(f0, f1, f2, (hi - lo) / Ngrids)
        variables["compress_var"][name] = {"srmin": np.float32(lo), "srmax": np.float32(hi),
                                           "poly_coeff": coeff.astype(np.float32)}
        # compression error on a 10x finer grid, in float64 (utils.py:283-290)
        x = np.linspace(lo, hi * (1 - 1e-6), Ngrids * 10 + 1)
        e0, e1, e2 = _embedding_jet(layers, x)
        delta = (hi - lo) / Ngrids
        idx = ((x - lo) / delta).astype(int)
        x0 = (x - lo - idx * delta)[:, None]
        c = coeff[np.clip(idx, 0, Ngrids - 1)]
        p0 = sum(c[:, i] * x0 ** (5 - i) for i in range(6))
        p1 = sum((5 - i) * c[:, i] * x0 ** (4 - i) for i in range(5))
        p2 = sum((5 - i) * (4 - i) * c[:, i] * x0 ** (3 - i) for i in range(4))
        for lst, a, b in zip(errs, (e0, e1, e2), (p0, p1, p2)):
            lst.append((a - b).reshape(-1))
    err = [np.concatenate(e) for e in errs]
    print("# Model Compressed: %d embedding nets, %d intervals" % (Y * Y, Ngrids))
    print("# Compression (0,1,2)-order error: Mean = (%.1e,%.1e,%.1e), Max = (%.1e,%.1e,%.1e)"
          % (err[0].mean(), err[1].mean(), err[2].mean(), err[0].max(), err[1].max(), err[2].max()))
    return model, variables


def periodic_replicate(n_copy, coord, box, type_idx=None, force=None, velocity=None):
    """Replicate a periodic system n_copy times along each axis
    (deepmd_jax/utils.py:299-327).  n_copy: scalar or (3,); coord (N, 3);
    box scalar, (3,) or (3, 3).  Returns [coord, box] plus the tiled
    type_idx, force and velocity that were given.  Copies along axis d are
    shifted by i * box[:, d] and stacked outermost, x first; the returned box
    is n_copy * box for a scalar or (3,) box, diag(n_copy) @ box for a
    matrix."""
    n_copy = (np.asarray(n_copy) * np.ones(3)).astype(int)
    box = np.array(box, dtype=float)
    if box.size <= 3:
        out_box = n_copy * box
        box = np.diag(box * np.ones(3))
    else:
        out_box = np.diag(n_copy) @ box
    coord = np.asarray(coord, dtype=float)
    for d in range(3):
        coord = np.concatenate([coord + i * box[:, d] for i in range(n_copy[d])]).reshape(-1, 3)
    ret = [coord, out_box]
    n = int(n_copy.prod())
    if type_idx is not None:
        ret.append(np.tile(type_idx, n))
    if force is not None:
        ret.append(np.concatenate([force] * n))
    if velocity is not None:
        ret.append(np.concatenate([velocity] * n))
    return ret
