"""The host predicate that decides whether an eps inversion may skip its
pivot guard (qx_eps_at_least_identity): eps(w) = I + B diag(chi'(w)) B^T >= I
needs every occupied level below every virtual one -- compared as min(virtual)
- max(occupied), since QP levels of an evGW iteration need not stay sorted --
and every real shift below that gap.  Host-only: runs without a GPU."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def lib():
    from quasix_b200 import _native
    return _native.load()


def cert(lib, e, nocc, wmax=0.0):
    e = np.ascontiguousarray(e, dtype=np.float64)
    return lib.qx_eps_at_least_identity(e.ctypes.data, nocc, e.shape[0] - nocc, float(wmax))


def test_sorted_levels(lib):
    e = np.array([-1.0, -0.5, 0.2, 0.9])
    assert cert(lib, e, 2) == 1
    assert cert(lib, e, 2, 0.69) == 1   # below the gap 0.7
    assert cert(lib, e, 2, 0.7) == 0    # at the gap chi' diverges
    assert cert(lib, e, 2, -0.5) == 1   # |w| counts


def test_unsorted_levels(lib):
    # The gap is min(virtual) - max(occupied), not e[nocc] - e[nocc-1].
    e = np.array([-0.2, -1.0, 0.5, 0.1])  # max occ -0.2, min vir 0.1: gap 0.3
    assert cert(lib, e, 2) == 1
    assert cert(lib, e, 2, 0.29) == 1
    assert cert(lib, e, 2, 0.31) == 0
    # e[nocc] - e[nocc-1] = 1.5 would wrongly certify a shift of 0.6.
    e = np.array([-1.0, -0.2, 1.3, 0.1])
    assert cert(lib, e, 2, 0.6) == 0


def test_crossed_or_degenerate_levels(lib):
    assert cert(lib, np.array([-1.0, 0.3, 0.2, 1.0]), 2) == 0   # occupied above a virtual
    assert cert(lib, np.array([-1.0, 0.2, 0.2, 1.0]), 2) == 0   # zero transition
    assert cert(lib, np.array([-1.0, np.nan, 0.2, 1.0]), 2) == 0
