"""compress_model (deepmd_jax/utils.py:250-297) on the CPU: the package's
float64 jet + closed-form quintics against (1) the fixture generator's
tables, built from the float64 oracle net with torch autograd, and (2)
scipy's BPoly.from_derivatives -> PPoly, the construction the reference
calls, fed with the oracle's values and derivatives.  Tolerance: float32
rounding: each term c_i x0^(5-i) at x0 = h (the interval width) agrees to
1e-6 of the net's largest value; the high-order coefficients themselves are
differences of nearly equal numbers divided by h^5, so they are compared as
these terms."""
import copy

import numpy as np
import torch

from make_golden import golden_models, hermite_compressed
from oracle import model as om


def test_compress_model_matches_fixture_tables_and_scipy():
    from scipy.interpolate import BPoly, PPoly
    from deepmd_jax_b200.utils import DPModelStub, compress_model
    p, v = golden_models()["B"]
    model = DPModelStub(copy.deepcopy(dict(p)))
    model, var = compress_model(model, copy.deepcopy(v), 256, 0.5)
    assert model.params["is_compressed"] is True
    _, vref = hermite_compressed(p, v, ngrids=256, rmin=0.5)
    nt = int(p["ntypes"])
    for k in range(nt * nt):
        name = "embedding_net_%d" % k
        got, ref = var["compress_var"][name], vref["compress_var"][name]
        assert got["poly_coeff"].shape == ref["poly_coeff"].shape == (256, 6, ref["poly_coeff"].shape[2])
        assert got["srmin"] == ref["srmin"] and got["srmax"] == ref["srmax"]
        _terms_close(got["poly_coeff"], ref["poly_coeff"], (float(ref["srmax"]) - float(ref["srmin"])) / 256, name)
    # scipy's construction on one net, values and derivatives from the oracle
    from deepmd_jax_b200.utils import sr
    m = om.OracleModel(dict(p) | {"is_compressed": False}, v, torch.float64)
    lo64 = (0.0 - float(p["sr_mean"][0])) / float(p["sr_std"][0])
    hi64 = (float(sr(0.5, float(p["rcut"]))) - float(p["sr_mean"][0])) / float(p["sr_std"][0])
    x = torch.linspace(lo64, hi64, 17, dtype=torch.float64).requires_grad_(True)
    f0 = m.embed(1, x)
    W = f0.shape[1]
    f1 = torch.stack([torch.autograd.grad(f0[:, w].sum(), x, create_graph=True)[0] for w in range(W)], 1)
    f2 = torch.stack([torch.autograd.grad(f1[:, w].sum(), x, retain_graph=True)[0] for w in range(W)], 1)
    xs = x.detach().numpy()
    poly = PPoly.from_bernstein_basis(BPoly.from_derivatives(
        xs, np.stack([f0.detach().numpy(), f1.detach().numpy(), f2.detach().numpy()], axis=1), orders=None))
    want = poly.c.transpose(1, 0, 2)
    p16 = DPModelStub(copy.deepcopy(dict(p)))
    _, v16 = compress_model(p16, copy.deepcopy(v), 16, 0.5)
    got = v16["compress_var"]["embedding_net_1"]["poly_coeff"]
    _terms_close(got, want, (hi64 - lo64) / 16, "scipy")


def _terms_close(got, want, h, name):
    powers = h ** (5 - np.arange(6))[None, :, None]
    err = np.abs(got.astype(np.float64) - want) * powers
    assert err.max() <= 1e-6 * np.abs(want[:, 5]).max(), (name, err.max())
