"""qx_screened_interaction_noalloc (scratch in a file-scope device array)
against qx_screened_interaction on the same inputs, through the C ABI.

Collected last on purpose: it must pass both in a fresh process and after
every other GPU test.  Tolerance: both paths run the same FP64 sweep, so Wc
agrees to 1e-12 relative (the Wc bar of the FP64 parity tests).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NAUX = 1024
MAX_NFREQ = 4096
TOL = 1e-12


def make_pi(nfreq, naux, seed):
    """Pi[w] = -X_w X_w^T * s_w: symmetric negative semidefinite, so I - Pi is SPD."""
    rng = np.random.default_rng(seed)
    k = max(8, naux // 3)
    x = rng.standard_normal((nfreq, naux, k)) / np.sqrt(k)
    s = np.linspace(2.0, 0.05, nfreq)[:, None, None]
    return np.ascontiguousarray(-np.einsum("wik,wjk->wij", x, x) * s)


@pytest.fixture(scope="module")
def env():
    import torch
    from quasix_b200 import _native
    import quasix_b200 as q
    return torch, _native.context(0), q


def noalloc(ctx, pi_dev, wc_dev):
    nfreq, naux = pi_dev.shape[0], pi_dev.shape[1]
    ctx.check(ctx.lib.qx_screened_interaction_noalloc(ctx.handle, nfreq, naux, C.c_void_p(pi_dev.data_ptr()),
                                                      C.c_void_p(wc_dev.data_ptr())))


def rel_err(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


@pytest.mark.parametrize("nfreq,naux", [(6, 300), (5, MAX_NAUX)])
def test_matches_screened_interaction_two_calls(env, nfreq, naux):
    torch, ctx, q = env
    for call, seed in enumerate((11, 12)):  # two calls in a row, different inputs
        pi = make_pi(nfreq, naux, seed + naux)
        ref = q.compute_epsilon_inverse_minus_identity(pi)
        pi_d = torch.from_numpy(pi).cuda()
        wc_d = torch.full_like(pi_d, float("nan"))
        torch.cuda.synchronize()
        noalloc(ctx, pi_d, wc_d)
        got = wc_d.cpu().numpy()
        assert np.isfinite(got).all(), call
        assert rel_err(got, ref) < TOL, (call, rel_err(got, ref))


def test_in_place_and_no_device_memory_growth(env):
    torch, ctx, q = env
    nfreq, naux = 7, 520
    pi = make_pi(nfreq, naux, 5)
    ref = q.compute_epsilon_inverse_minus_identity(pi)
    buf = torch.from_numpy(pi).cuda()
    first = buf.clone()
    torch.cuda.synchronize()
    noalloc(ctx, first, first)  # pi and wc alias
    assert rel_err(first.cpu().numpy(), ref) < TOL
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    noalloc(ctx, buf, buf)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    assert rel_err(buf.cpu().numpy(), ref) < TOL


def test_rejects_sizes_beyond_the_limit_and_host_pointers(env):
    torch, ctx, q = env
    from quasix_b200._native import QxValueError
    big = torch.zeros((1, MAX_NAUX + 1, MAX_NAUX + 1), dtype=torch.float64, device="cuda")
    with pytest.raises(QxValueError, match="naux <= 1024"):
        noalloc(ctx, big, big)
    small = torch.zeros((1, 8, 8), dtype=torch.float64, device="cuda")
    st = ctx.lib.qx_screened_interaction_noalloc(ctx.handle, MAX_NFREQ + 1, 8, C.c_void_p(small.data_ptr()),
                                                 C.c_void_p(small.data_ptr()))
    assert st == 1 and b"nfreq <= 4096" in ctx.lib.qx_last_error(ctx.handle)
    host = np.zeros((1, 8, 8))
    st = ctx.lib.qx_screened_interaction_noalloc(ctx.handle, 1, 8, C.c_void_p(host.ctypes.data),
                                                 C.c_void_p(host.ctypes.data))
    assert st == 1 and b"device pointers" in ctx.lib.qx_last_error(ctx.handle)
