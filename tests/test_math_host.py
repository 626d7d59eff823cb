"""CPU check of the per-particle math shared by the CUDA kernels
(diffcp_b200/csrc/cloth_math.cuh, compiled here with g++ through
tests/native/math_harness.cpp) against the oracle and torch.autograd."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle import sim64

HERE = os.path.dirname(os.path.abspath(__file__))
_dbl = ctypes.POINTER(ctypes.c_double)
_int = ctypes.POINTER(ctypes.c_int)


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("harness") / "math_harness.so")
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-Wno-unknown-pragmas", "-o", out,
                    os.path.join(HERE, "native", "math_harness.cpp")], check=True)
    return ctypes.CDLL(out)


def _p(a):
    return a.ctypes.data_as(_dbl)


def _random_F(n, seed):
    rng = np.random.default_rng(seed)
    F = np.eye(3)[None] + 0.15 * rng.standard_normal((n, 3, 3))
    F[: n // 4, :, 2] *= 0.8                      # normal compression (R22 <= 1 branch)
    F[n // 4: n // 2, :, 2] *= 1.3                # stretched normal
    F[-3] = np.eye(3)                             # exactly degenerate in-plane SVD
    th = 0.3
    F[-2] = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
    F[-1] = np.diag([1.0 + 1e-5, 1.0 - 1e-5, 0.97])   # near-degenerate
    return F


def _mu_la(E, nu):
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


def test_stress_forward_matches_oracle(lib):
    n = 64
    F = _random_F(n, 0)
    E, nu, ks, kc = 5e3, 0.3, 120.0, 340.0
    mu, la = _mu_la(E, nu)
    prm = np.tile([mu, la, ks, kc], (n, 1)).astype(np.float64)
    P = np.zeros((n, 3, 3))
    lib.h_stress_fwd(n, 1, _p(np.ascontiguousarray(F)), _p(prm), _p(P))
    d = torch.float64
    ref = sim64.triangle_stress(torch.tensor(F), torch.tensor(E, dtype=d), torch.tensor(nu, dtype=d),
                                torch.tensor(ks, dtype=d), torch.tensor(kc, dtype=d)).numpy()
    np.testing.assert_allclose(P, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    Pf = np.zeros((n, 3, 3))
    lib.h_stress_fwd(n, 0, _p(np.ascontiguousarray(F)), _p(prm), _p(Pf))
    assert np.abs(Pf - ref).max() <= 2e-5 * np.abs(ref).max()


@pytest.mark.parametrize("mode", ["exact", "reference"])
@pytest.mark.parametrize("dbl", [1, 0])
def test_stress_adjoint_matches_autograd(lib, mode, dbl):
    n = 64
    F = _random_F(n, 1)
    rng = np.random.default_rng(2)
    gP = rng.standard_normal((n, 3, 3))
    E0, nu0, ks0, kc0 = 5e3, 0.3, 120.0, 340.0
    Ft = torch.tensor(F, requires_grad=True)
    d = torch.float64
    E = torch.tensor(E0, dtype=d, requires_grad=True)
    nu = torch.tensor(nu0, dtype=d, requires_grad=True)
    ks = torch.tensor(ks0, dtype=d, requires_grad=True)
    kc = torch.tensor(kc0, dtype=d, requires_grad=True)
    P = sim64.triangle_stress(Ft, E, nu, ks, kc, svd_grad=mode)
    (P * torch.tensor(gP)).sum().backward()
    mu, la = _mu_la(E0, nu0)
    prm = np.tile([mu, la, ks0, kc0], (n, 1)).astype(np.float64)
    gF = np.zeros((n, 3, 3))
    gprm = np.zeros((n, 4))
    lib.h_stress_bwd(n, dbl, _p(np.ascontiguousarray(F)), _p(prm), _p(np.ascontiguousarray(gP)),
                     0 if mode == "exact" else 1, _p(gF), _p(gprm))
    ref = Ft.grad.numpy()
    tol = 1e-8 if dbl else 3e-4
    scale = np.abs(ref).max(axis=(1, 2), keepdims=True) + 1.0
    err = np.abs(gF - ref) / scale
    assert err.max() < tol, (np.unravel_index(err.argmax(), err.shape), err.max())
    gmu, gla = gprm[:, 0].sum(), gprm[:, 1].sum()
    dmu_dE, dmu_dnu = 1 / (2 * (1 + nu0)), -E0 / (2 * (1 + nu0) ** 2)
    D = (1 + nu0) * (1 - 2 * nu0)
    dla_dE, dla_dnu = nu0 / D, E0 * (1 + 2 * nu0 ** 2) / D ** 2
    gE = gmu * dmu_dE + gla * dla_dE
    gnu = gmu * dmu_dnu + gla * dla_dnu
    rt = 1e-8 if dbl else 2e-4
    assert gE == pytest.approx(float(E.grad), rel=rt)
    assert gnu == pytest.approx(float(nu.grad), rel=rt)
    assert gprm[:, 2].sum() == pytest.approx(float(ks.grad), rel=rt)
    assert gprm[:, 3].sum() == pytest.approx(float(kc.grad), rel=rt)


def test_svd2_and_clamped_backward_match_oracle(lib):
    rng = np.random.default_rng(5)
    n = 40
    A = np.eye(2)[None] + 0.4 * rng.standard_normal((n, 2, 2))
    A[0] = np.eye(2)
    A[1] = np.array([[1.0, 2e-6], [0.0, 1.0]])
    U = np.zeros((n, 2, 2)); S = np.zeros((n, 2)); V = np.zeros((n, 2, 2))
    lib.h_svd2(n, _p(np.ascontiguousarray(A)), _p(U), _p(S), _p(V))
    Ur, Sr, Vr = sim64.svd2_taichi(torch.tensor(A))
    np.testing.assert_allclose(U, Ur.numpy(), atol=1e-12)
    np.testing.assert_allclose(S, np.diagonal(Sr.numpy(), axis1=1, axis2=2), atol=1e-12)
    np.testing.assert_allclose(V, Vr.numpy(), atol=1e-12)
    gU = rng.standard_normal((n, 2, 2)); gV = rng.standard_normal((n, 2, 2))
    gA = np.zeros((n, 2, 2))
    lib.h_svd2_bwd(n, _p(gU), _p(gV), _p(U), _p(S), _p(V), _p(gA))
    ref = sim64.svd_backward_clamped(torch.tensor(gU), torch.zeros(n, 2, 2, dtype=torch.float64), torch.tensor(gV), Ur, Sr, Vr).numpy()
    np.testing.assert_allclose(gA, ref, rtol=1e-10, atol=1e-8)


@pytest.mark.parametrize("mu", [0.0, 0.4])
def test_grid_bc_forward_and_adjoint(lib, mu):
    rng = np.random.default_rng(9)
    G, bound = 16, 3
    n = 400
    ijk = rng.integers(0, G, size=(n, 3)).astype(np.int32)
    ijk[: n // 2, 1] = rng.integers(0, bound, size=n // 2)   # many floor nodes
    v = rng.standard_normal((n, 3))
    v[:20, [0, 2]] *= 1e-22          # floor nodes with a denormal tangential speed
    v[:20, 1] = -np.abs(v[:20, 1])
    ijk[:20, 1] = 0
    out = np.zeros((n, 3))
    lib.h_grid_bc(n, _p(v), ijk.ctypes.data_as(_int), G, bound, ctypes.c_double(mu), _p(out))
    vt = torch.tensor(v, requires_grad=True)
    mut = torch.tensor(mu, dtype=torch.float64, requires_grad=True)
    m = torch.ones(n, dtype=torch.float64)
    ref = sim64.grid_op(vt * (m[:, None] + 1e-9), m, torch.tensor(ijk, dtype=torch.long), G, bound, friction=mut)
    np.testing.assert_allclose(out, ref.detach().numpy(), rtol=1e-12, atol=1e-12)
    gout = rng.standard_normal((n, 3))
    (ref * torch.tensor(gout)).sum().backward()
    gv = np.zeros((n, 3))
    gmu = np.zeros(n)
    lib.h_grid_bc_bwd(n, _p(v), ijk.ctypes.data_as(_int), G, bound, ctypes.c_double(mu), _p(gout), _p(gv), _p(gmu))
    assert np.isfinite(gv).all() and np.isfinite(gmu).all()
    ok = np.isfinite(vt.grad.numpy()).all(axis=1)
    np.testing.assert_allclose(gv[ok], vt.grad.numpy()[ok], rtol=1e-9, atol=1e-9)
    if np.isfinite(float(mut.grad)):
        assert gmu.sum() == pytest.approx(float(mut.grad), rel=1e-9, abs=1e-12)


@pytest.mark.parametrize("mode", ["exact", "reference"])
def test_float_stress_keeps_precision_at_small_strain(lib, mode):
    """Cloth strains are ~1e-5..1e-3: the float build, fed F - I, must keep
    near-float relative precision in P and in dL/d(mu, la) instead of losing it
    to cancellation of O(1) numbers."""
    n = 64
    rng = np.random.default_rng(7)
    F = np.eye(3)[None] + 1e-4 * rng.standard_normal((n, 3, 3))
    F[: n // 2, 2, 2] -= 3e-4                      # normal compression: contact branch
    E0, nu0, ks0, kc0 = 5e3, 0.3, 120.0, 340.0
    mu, la = _mu_la(E0, nu0)
    prm = np.tile([mu, la, ks0, kc0], (n, 1)).astype(np.float64)
    Pd = np.zeros((n, 3, 3)); Pf = np.zeros((n, 3, 3))
    lib.h_stress_fwd(n, 1, _p(np.ascontiguousarray(F)), _p(prm), _p(Pd))
    lib.h_stress_fwd(n, 0, _p(np.ascontiguousarray(F)), _p(prm), _p(Pf))
    assert np.abs(Pf - Pd).max() <= 2e-5 * np.abs(Pd).max()
    gP = rng.standard_normal((n, 3, 3))
    gd = np.zeros((n, 4)); gf = np.zeros((n, 4)); gF = np.zeros((n, 3, 3))
    m = 0 if mode == "exact" else 1
    lib.h_stress_bwd(n, 1, _p(np.ascontiguousarray(F)), _p(prm), _p(gP), m, _p(gF), _p(gd))
    lib.h_stress_bwd(n, 0, _p(np.ascontiguousarray(F)), _p(prm), _p(gP), m, _p(gF), _p(gf))
    for j in range(4):
        assert abs(gf[:, j].sum() - gd[:, j].sum()) <= 1e-5 * np.abs(gd[:, j]).sum() + 1e-30, j


def test_float_stress_stays_finite_on_nearly_collapsed_columns(lib):
    """Deformation gradients with one column almost collapsed (|h|^2 far below
    1, as in a cloth crumpled hard): the float build's QR must sum those squared
    norms from components (the small-strain identity 1 + (|h|^2 - 1) can round
    below zero there) and give the double build's stress."""
    rng = np.random.default_rng(21)
    F = []
    for k in range(300):
        A = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        c = k % 3
        if c == 0:
            A[:, 0] *= 10.0 ** rng.uniform(-3.5, -1)                           # short first column
        elif c == 1:
            A[:, 1] = A[:, 0] * rng.uniform(0.5, 2) + 10.0 ** rng.uniform(-3.5, -1) * rng.standard_normal(3)
        else:                                                                # third column nearly in-plane
            A[:, 2] = rng.standard_normal(2) @ A[:, :2].T + 10.0 ** rng.uniform(-3.5, -1) * rng.standard_normal(3)
        F.append(A)
    F = np.ascontiguousarray(np.stack(F))
    n = len(F)
    prm = np.tile([300.0, 200.0, 100.0, 100.0], (n, 1))
    P32, P64 = np.zeros((n, 9)), np.zeros((n, 9))
    lib.h_stress_fwd(n, 0, _p(F), _p(prm), _p(P32))
    lib.h_stress_fwd(n, 1, _p(F), _p(prm), _p(P64))
    assert np.isfinite(P32).all()
    # smallest singular values down to 1e-5: the stress's condition number
    # reaches 1e5, and float32 keeps a few 1e-3 of it
    scale = np.abs(P64).max(axis=1)
    assert (np.abs(P32 - P64).max(axis=1) <= 1e-2 * scale).all()
