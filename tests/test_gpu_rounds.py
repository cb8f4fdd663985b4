"""The mixed form in rounds (chord kernel, Hessians on the tensor cores or on
CUDA cores, inverses) on the 2-D Euler closure (needs a B200).

1. The re-factorisation's inverse Hessian H^-1 (FP32) of both Hessian forms
   against H^-1 of the FP64 Hessian computed here from the basis tables and
   the Euler ansatz's DU (closure.cpp:255-271: H(m nT + j, l nT + i) =
   sum_k phi_kj phi_ki wt_k DU_ml(Lambda_k)). The tensor-core form splits Q and
   DU into high and low BF16 parts (relative error about 2^-16 per product);
   the bound, 2e-3 relative in the Frobenius norm, leaves room for the FP32
   Cholesky of Hessians with condition numbers up to about 1e4.
2. Time steps in every form against the FP64 oracle, within the mixed bound
   (relative L1 1e-6 of moments and of mean/variance).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from uqcreator_b200 import Solver, workloads as W, MIXED

from ._util import rel_l1

pytestmark = pytest.mark.gpu


def _euler_du(L, gamma=1.4):
    """EulerClosure2D::DU (eulerclosure2d.cpp:54-88), packed upper order
    (0,0)(0,1)(0,2)(0,3)(1,1)(1,2)(1,3)(2,2)(2,3)(3,3), as physics.cuh writes it."""
    g = -gamma
    A = 1.0 / (1.0 - gamma)
    v1, v2, v3, v4 = L
    i4 = 1.0 / v4
    q = (v2 * v2 + v3 * v3 - 2 * v1 * v4 - 2 * v4 * g) * (0.5 * i4)
    e = A * np.exp(A * (q + np.log(-v4)))
    vt = e * (v2 * v2 + v3 * v3 + 2 * v4 * g) * (0.5 * i4 ** 3)
    return np.array([-e, v2 * e * i4, v3 * e * i4, -(0.5 * (v2 * v2 + v3 * v3 - 2 * v4) * e) * i4 ** 2,
                     -(e * (v2 * v2 + (g + 1) * v4)) * i4 ** 2, -(v2 * v3 * e) * i4 ** 2, v2 * vt,
                     -(e * (v3 * v3 + (g + 1) * v4)) * i4 ** 2, v3 * vt,
                     -e * (v2 ** 4 + v3 ** 4 + 4 * v3 * v3 * v4 * g - 4 * v4 * v4 * g + 2 * v2 * v2 * (v3 * v3 + 2 * v4 * g))
                     * (0.25 * i4 ** 4)])


def _fp64_hessian(phi, w, dim_xi, lam):
    nq, nt = phi.shape
    wt = w / 2.0 ** dim_xi
    Lam = lam @ phi.T                      # (4, nq)
    du = np.array([_euler_du(Lam[:, k]) for k in range(nq)])    # (nq, 10)
    H = np.zeros((4 * nt, 4 * nt))
    b = 0
    for m in range(4):
        for l in range(m, 4):
            blk = (phi * (wt * du[:, b])[:, None]).T @ phi
            H[m * nt:(m + 1) * nt, l * nt:(l + 1) * nt] = blk
            H[l * nt:(l + 1) * nt, m * nt:(m + 1) * nt] = blk.T
            b += 1
    return H


def _state_after_steps(toml, steps=2):
    s = Solver(toml)
    s.init_state()
    s.step(steps)
    return s


def test_default_form_uses_tensor_cores():
    s = Solver(W.euler2d(nx=8, ny=3))
    s.set_precision(MIXED)
    f = s.form()
    assert f["mixed_form"] == 2 and f["mixed_rounds"] >= 1


@pytest.mark.parametrize("form", [1, 2], ids=["cuda_cores", "tensor_cores"])
def test_reformed_inverse_matches_fp64(form):
    toml = W.euler2d(nx=16, ny=4)
    s = _state_after_steps(toml)
    _, lam, _ = s.download_state()
    phi, _, _, w = s.tables()
    cells = np.arange(0, s.n_cells, 3)
    got = s.debug_mixed_inverse(cells, form)
    worst = 0.0
    for c, hinv in zip(cells, got):
        ref = np.linalg.inv(_fp64_hessian(phi, w, s.dim_xi, lam[c]))
        assert np.isfinite(hinv).all()
        np.testing.assert_allclose(hinv, hinv.T, rtol=0, atol=1e-6 * np.abs(hinv).max())
        worst = max(worst, np.linalg.norm(hinv - ref) / np.linalg.norm(ref))
    assert worst <= 2e-3, worst


def test_tensor_and_cuda_core_inverses_agree():
    s = _state_after_steps(W.euler2d(nx=12, ny=4, degree=3, nquad=6))
    cells = np.arange(s.n_cells)
    a = s.debug_mixed_inverse(cells, 1)
    b = s.debug_mixed_inverse(cells, 2)
    rel = np.linalg.norm((a - b).reshape(len(cells), -1), axis=1) / np.linalg.norm(a.reshape(len(cells), -1), axis=1)
    assert rel.max() <= 2e-3, rel.max()


@pytest.mark.parametrize("form", [0, 1, 2], ids=["single_kernel", "rounds_cuda_cores", "rounds_tensor_cores"])
@pytest.mark.parametrize("rounds", [1, 3])
def test_rounds_match_oracle(form, rounds):
    toml = W.euler2d(nx=24, ny=5)
    s = Solver(toml)
    s.set_precision(MIXED)
    s.set_option("mixed_hessian", form)
    s.set_option("mixed_rounds", rounds)
    assert s.form()["mixed_form"] == form
    o = Oracle(toml, W.mesh_for(toml))
    s.init_state(); o.init_state()
    info = s.step(5)
    o.step(5)
    assert info["failed_cells"] == 0 and info["steps"] == 5
    us, _, _ = s.download_state()
    uo, _, _ = o.get_state()
    assert float(np.abs(us - uo).sum() / np.abs(uo).sum()) <= 1e-6
    err = rel_l1(s.mean_var(), o.mean_var(), o.geometry()["area"])
    assert np.all(err <= 1e-6), err


def test_rounds_are_reproducible_and_keep_inverses():
    """Held inverses persist across steps (the second run of steps needs fewer
    re-factorisations than a cold start) and a state uploaded again starts
    cold, so the same steps give the same result."""
    toml = W.euler2d(nx=20, ny=5)
    s = Solver(toml); s.init_state(); s.step(2)
    s.set_precision(MIXED)
    u0, l0, v0 = s.download_state()
    a = s.step(3)
    ua = s.download_state()[0]
    s.upload_state(u0, l0, v0)
    b = s.step(3)
    ub = s.download_state()[0]
    assert a["newton_iterations"] == b["newton_iterations"]
    np.testing.assert_array_equal(ua, ub)
