"""Known-answer test of the tcgen05 / TMEM path (descriptors, instruction
descriptor, allocation, commit/wait, TMEM loads): exact BF16 products."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [0, 1])
def test_tcgen05_known_answer(variant):
    from deepmd_jax_b200 import _lib
    lib = _lib.load()
    lib.dpb_selftest_tcgen05.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    out = torch.zeros(128 * 64, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.dpb_selftest_tcgen05(variant, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(err.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    m, k, n = np.arange(128)[:, None], np.arange(32)[None, :], np.arange(64)
    A = ((m * 3 + k * 5) % 17 - 8) / 8.0
    B = ((np.arange(32)[:, None] * 7 + n[None, :] * 11) % 13 - 6) / 4.0
    assert np.array_equal(out.cpu().numpy().reshape(128, 64), A @ B)
