"""The C-ABI library loads and exports every symbol include/qx_gw.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(qx_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["qx_ctx_create", "qx_get_sigma_diag", "qx_evgw", "qx_bse_davidson", "qx_g0w0_cd"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from quasix_b200 import _native
    lib = _native.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # ctypes signatures cover every declared symbol.
    assert set(declared_functions()) <= set(_native.SIGNATURES)


def test_no_device_is_reported_cleanly():
    """Without a GPU the context creation returns QX_ERR_NO_DEVICE, it does not crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from quasix_b200 import _native
    with pytest.raises(_native.QxError):
        _native.Context(0)


def test_host_only_entry_points():
    """Pure host entry points work without a GPU and match the oracle."""
    import numpy as np
    from oracle import qx_oracle as O
    import quasix_b200 as q
    for nw in (1, 2, 16, 32, 48):
        f, w = q.get_scaled_legendre_roots(nw, 0.5)
        f2, w2 = O.get_scaled_legendre_roots(nw, 0.5)
        assert np.allclose(f, f2, rtol=1e-11, atol=0) and np.allclose(w, w2, rtol=1e-11, atol=0)
