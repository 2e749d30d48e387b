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
    """Any other flax class the pickle mentions (module bookkeeping)."""

    def __init__(self, *a, **k):
        pass

    def __setstate__(self, state):
        if isinstance(state, dict):
            self.__dict__.update(state)


def _reconstruct_array(fun, args, arr_state, aval_state):
    """Stand-in for jax._src.array._reconstruct_array: returns numpy."""
    a = fun(*args)
    a.__setstate__(arr_state)
    return np.asarray(a)


def _frozen_dict(*args, **kw):
    d = dict(*args, **kw)
    return d


class _Unpickler(pickle.Unpickler):
    def find_class(self, module, name):
        if module.startswith("deepmd_jax") and name == "DPModel":
            return DPModelStub
        if module.startswith("jax") and name in ("_reconstruct_array",):
            return _reconstruct_array
        if module.startswith("jax") and "Array" in name:
            return np.asarray
        if module.startswith("flax") and name == "FrozenDict":
            return _frozen_dict
        if module.startswith("flax") or module.startswith("jax"):
            return _Opaque
        if module.startswith(("numpy", "builtins", "collections", "copyreg", "_codecs")):
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
