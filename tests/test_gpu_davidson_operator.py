"""davidson_bse with a caller-supplied operator (bse/davidson.rs:372-508)
against the oracle's Davidson and dense eigh, and against the BSE kernel's own
solve when the operator is that kernel's matvec."""
import numpy as np
import pytest

from oracle import qx_oracle as O

pytestmark = pytest.mark.gpu


def dense_operator(n, seed):
    rng = np.random.default_rng(seed)
    gaps = np.sort(rng.uniform(0.3, 3.0, n))
    c = rng.standard_normal((n, n)) * 0.01
    return gaps, np.diag(gaps) + 0.5 * (c + c.T)


@pytest.mark.parametrize("tensors", ["numpy", "torch"])
def test_callback_davidson_matches_oracle_and_eigh(tensors):
    import torch
    import quasix_b200 as q
    n = 240
    gaps, h = dense_operator(n, 2)
    ht = torch.as_tensor(h, device="cuda")
    op = (lambda x: h @ x) if tensors == "numpy" else (lambda x: ht @ x)
    cfg = q.DavidsonConfig(n_roots=4, max_iter=200, max_space=40, tol_residual=1e-9)
    got = q.davidson_bse(op, gaps, cfg, tensors=tensors)
    ref = O.davidson_bse(lambda x: h @ x, gaps, O.DavidsonConfig(n_roots=4, max_iter=200, max_space=40,
                                                                 tol_residual=1e-9))
    exact = np.linalg.eigvalsh(h)[:4]
    assert got["all_converged"]
    assert np.abs(got["eigenvalues"] - exact).max() < 1e-9
    assert np.abs(got["eigenvalues"] - ref["eigenvalues"]).max() < 1e-9
    for j in range(4):
        v = got["eigenvectors"][:, j]
        assert np.linalg.norm(h @ v - got["eigenvalues"][j] * v) < 1e-8


def test_callback_davidson_equals_kernel_solve():
    import quasix_b200 as q
    from quasix_b200.synth import bse_blocks, make_system
    s = make_system(6, 30, 90, seed=5, pi_norm=2.0)
    dia, dij, dab = bse_blocks(s.lpq, 6)
    w0 = q.bse.screened_w0(s.mo_energy, np.ascontiguousarray(s.lpq[:, :6, 6:]))
    delta = (s.mo_energy[None, 6:] - s.mo_energy[:6, None]).reshape(-1)
    k = q.BSETDAKernel(6, 30, 90, delta, dia, dij, dab, w0)
    cfg = q.DavidsonConfig(n_roots=3, max_iter=100, tol_residual=1e-8)
    own = k.solve_davidson_with_config(cfg)
    cb = q.davidson_bse(k.apply_hamiltonian_batch, delta, cfg)
    k.close()
    assert cb["iterations"] == own["iterations"]
    assert np.abs(cb["eigenvalues"] - own["eigenvalues"]).max() < 1e-12


def test_callback_errors_propagate():
    import quasix_b200 as q
    gaps, h = dense_operator(50, 3)

    def bad(x):
        raise KeyError("operator failed")

    with pytest.raises(KeyError):
        q.davidson_bse(bad, gaps, q.DavidsonConfig(n_roots=2))
    with pytest.raises(ValueError):
        q.davidson_bse(lambda x: x[:-1], gaps, q.DavidsonConfig(n_roots=2))
