"""CPU: the oracle's trust-region Newton path and deflation bias
(solver_rtr.hpp:30-459) against the properties the reference's own tests check
(tests/test_solver_rtr.py, tests/test_deflation.py): the Hessian-vector product
against finite differences of the gradient, the deflation bias against its
closed form and gradient identity, and Newton solves that reach the CG / SCF
solution, conserve particles and honour the projector.
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy.linalg import expm

import newton_cases as nc
from conftest import herm
from oracle import native_np as nn


def _offdiag(X):
    X = X.copy()
    i = np.arange(X.shape[-1])
    X[..., i, i] = 0.0
    return X


def _skew(X):
    return 0.5 * (X - np.conj(np.swapaxes(X, -1, -2)))


def _expm_batch(A):
    s = A.shape
    return np.stack([expm(a) for a in A.reshape(-1, s[-2], s[-1])]).reshape(s)


def hvp_fd_errors(mod, args, seed=1):
    """Relative error of the joint HVP against forward differences of the
    gradient at two step sizes (the check of test_solver_rtr.py:77-135)."""
    T = float(args["T"])
    h = args["h"]
    w2 = args["w2d"]
    nb = h.shape[-1]

    def fock(P):
        return np.asarray(mod.build_fock_apply(args, np.ascontiguousarray(P, np.complex128), None)[2])

    def ft(Q, M):
        return np.conj(np.swapaxes(Q, -1, -2)) @ M @ Q

    def dens(Q, p):
        return (Q * p[..., None, :]) @ np.conj(np.swapaxes(Q, -1, -2))

    rng = np.random.default_rng(seed)
    eps, Q = np.linalg.eigh(fock(np.zeros_like(h)))
    X0 = _skew(_offdiag(rng.standard_normal(Q.shape) + 1j * rng.standard_normal(Q.shape)))
    Q = Q @ _expm_batch(0.2 * X0)
    p = np.clip(1.0 / (1 + np.exp((eps - np.median(eps)) / T)), 0.05, 0.95)
    mu = float(np.median(eps))

    def grad(Q, p):
        Ft = ft(Q, fock(dens(Q, p)))
        GQ = _offdiag((p[..., None, :] - p[..., :, None]) * Ft)
        gp = np.real(np.diagonal(Ft, axis1=-2, axis2=-1)) + T * np.log(p / (1 - p)) - mu
        return GQ, gp, Ft

    GQ, gp, Ft = grad(Q, p)
    X = _skew(_offdiag(rng.standard_normal(Q.shape) + 1j * rng.standard_normal(Q.shape)))
    dp = rng.standard_normal(p.shape) * 0.1
    HX, Hp = mod._rtr_joint_hvp(args, np.ascontiguousarray(X), np.ascontiguousarray(dp), np.ascontiguousarray(Q),
                                np.ascontiguousarray(p), np.ascontiguousarray(Ft))
    HX, Hp = np.asarray(HX), np.asarray(Hp)
    eQ, ep = [], []
    for e in (1e-5, 1e-6):
        GQe, gpe, _ = grad(Q @ _expm_batch(e * X), p + e * dp)
        fdQ = (GQe - GQ) / e
        fdp = (gpe - gp) / e
        fdp = fdp - np.sum(w2[..., None] * fdp) / (np.sum(w2) * nb)
        eQ.append(np.max(np.abs(fdQ - HX)) / max(np.max(np.abs(HX)), 1e-30))
        ep.append(np.max(np.abs(fdp - Hp)) / max(np.max(np.abs(Hp)), 1e-30))
    return eQ, ep, (X, dp, Q, p, Ft)


def test_joint_hvp_matches_finite_differences():
    args, _h = nc.multiband(5, 5, 0.05, 0.4, 4)
    eQ, ep, _ = hvp_fd_errors(nn, args)
    assert eQ[1] < 1e-4 and ep[1] < 1e-4
    assert eQ[1] < 0.2 * eQ[0] + 1e-12 and ep[1] < 0.2 * ep[0] + 1e-12


def test_deflation_bias_closed_form_and_gradient_identity():
    rng = np.random.default_rng(0)
    nk, nb = 2, 2
    w2d = np.arange(nk * nk).reshape(nk, nk).astype(np.float64) + 1.0
    sigma, length = 0.7, 0.5

    def rh(shape):
        return herm(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))

    P = rh((nk, nk, nb, nb))
    targets = np.stack([rh((nk, nk, nb, nb)) for _ in range(2)])
    Phi, S_pen, diag = nn._deflation_bias(P, targets, w2d, sigma, length)
    dP = rh((nk, nk, nb, nb))
    analytic = float(np.sum(w2d[..., None, None] * np.real(np.conj(S_pen) * dP)))
    fd = [(nn._deflation_bias(P + e * dP, targets, w2d, sigma, length)[0]
           - nn._deflation_bias(P - e * dP, targets, w2d, sigma, length)[0]) / (2 * e) for e in (1e-4, 1e-5)]
    assert abs(fd[1] - analytic) < 1e-4 * (abs(analytic) + 1.0)
    inv2L2 = 1.0 / (2.0 * length * length)
    d2 = np.array([np.sum(w2d[..., None, None] * np.abs(P - t) ** 2) for t in targets])
    phi = sigma * np.exp(-d2 * inv2L2)
    assert abs(Phi - np.sum(phi)) < 1e-12
    assert abs(diag - 2.0 * np.sum(-phi * inv2L2)) < 1e-12
    Phi0, S0, d0 = nn._deflation_bias(P, np.empty((0, nk, nk, nb, nb), np.complex128), w2d, 1.0, 1.0)
    assert Phi0 == 0.0 and d0 == 0.0 and np.max(np.abs(S0)) == 0.0


def test_newton_matches_cg_on_unique_minimum():
    args, h = nc.contact(g=0.3, nk=2)
    P0 = np.zeros_like(h)
    cg = nc.solve(nn, args, P0, 4.0, max_iter=400, tol_E=1e-10)
    nw = nc.solve(nn, args, P0, 4.0, max_iter=200, tol_grad=1e-7, optimizer="newton")
    assert nw["converged"]
    assert abs(nw["energy"] - cg["energy"]) < 1e-6


def test_newton_stationary_and_conserves_particles():
    args, h = nc.multiband(4, 4, 0.05, 0.3, 7)
    ne = 4 * 4 * 4 * 0.5
    r = nc.solve(nn, args, np.zeros_like(h), ne, max_iter=200, tol_grad=1e-6, optimizer="newton")
    assert r["converged"]
    assert nc.comm_rms(r["fock"], r["density"], args["w2d"]) < 1e-4
    assert abs(float(np.sum(args["w2d"][..., None] * r["p"])) - ne) < 1e-4


def test_newton_projector_and_deflation_noop():
    args, h = nc.hybridized(nk=2, ex=0.25)
    P0 = np.zeros_like(h)
    r = nc.solve(nn, args, P0, 4.0, optimizer="newton", tol_grad=1e-6, project_fn=nc.diag_projector)
    assert np.max(np.abs(r["density"][..., 0, 1])) < 1e-8
    r0 = nc.solve(nn, args, P0, 4.0, optimizer="newton", tol_grad=1e-6)
    assert np.max(np.abs(r0["density"][..., 0, 1])) > 1e-3
    r3 = nc.solve(nn, args, P0, 4.0, optimizer="newton", tol_grad=1e-6, deflation_targets=r0["density"][None],
                  deflation_sigma=0.0)
    np.testing.assert_array_equal(r3["density"], r0["density"])


def deflated_second_solution(mod, args, h):
    """The loop of solve_deflated (deflation.py:99-170) for a second solution:
    bias around the first, re-solve from a perturbed seed, re-polish unbiased,
    escalate the bias height by 3 until the result is a distinct basin."""
    P0 = np.zeros_like(h)
    w2d = args["w2d"]
    base = dict(optimizer="newton", tol_grad=1e-6, max_iter=300)
    r0 = nc.solve(mod, args, P0, 1.0, **base)
    length = 0.5 * float(np.sqrt(np.sum(w2d * np.sum(np.abs(r0["density"]) ** 2, axis=(-2, -1)))))
    sigma = max(abs(float(r0["energy"])), 1.0)
    rng = np.random.default_rng(0)
    for attempt in range(4):
        A = rng.standard_normal(P0.shape) + 1j * rng.standard_normal(P0.shape)
        seed = P0 + 1e-2 * (attempt + 1) * herm(A)
        rb = nc.solve(mod, args, seed, 1.0, deflation_targets=r0["density"][None], deflation_sigma=sigma,
                      deflation_length=length, **base)
        r1 = nc.solve(mod, args, rb["density"], 1.0, **base)
        dist = float(np.sqrt(np.sum(w2d * np.sum(np.abs(r1["density"] - r0["density"]) ** 2, axis=(-2, -1)))))
        if r1["converged"] and dist > 0.25 * length:
            return r0, rb, r1, attempt
        sigma *= 3.0
    return r0, rb, r1, None


def test_deflated_newton_reaches_the_metastable_solution():
    """Deflation moves the bistable model from its ground state (E = -delta - ex/2
    = -0.6) to the other solution (E = +delta - ex/2 = -0.4)."""
    args, h = nc.bistable()
    r0, _rb, r1, attempt = deflated_second_solution(nn, args, h)
    assert attempt is not None
    assert abs(r0["energy"] + 0.6) < 2e-2
    assert r1["converged"] and abs(r1["energy"] + 0.4) < 3e-2
    assert np.max(np.abs(r1["density"] - r0["density"])) > 1e-2


def test_newton_rejects_short_deflation_buffer():
    args, h = nc.hybridized(nk=2)
    with pytest.raises(ValueError):
        nn.solve_dm(args, np.zeros_like(h), 4.0, 10, 1e-7, 1e-6, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 1, 0.5, 20,
                    np.zeros((1, 2, 2, 2, 1), np.complex128), 1.0, 1.0, [], None, True, True, True)
