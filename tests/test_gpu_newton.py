"""GPU parity of the trust-region Newton path (optimizer=1, solver_rtr.hpp:30-459):
the joint Hessian-vector product and the deflation bias against the oracle and
against finite differences, and Newton solves (plain, projected, deflated)
against the oracle's solves on the problems of the reference's Newton and
deflation tests plus larger synthetic meshes."""

from __future__ import annotations

import numpy as np
import pytest

import newton_cases as nc
from conftest import herm
from cpp_hf_b200 import workloads
from test_oracle_newton import deflated_second_solution, hvp_fd_errors

pytestmark = pytest.mark.gpu


def test_joint_hvp_matches_oracle_and_finite_differences(native, oracle):
    args, _h = nc.multiband(5, 5, 0.05, 0.4, 4)
    eQ, ep, (X, dp, Q, p, Ft) = hvp_fd_errors(native, args)
    assert eQ[1] < 1e-4 and ep[1] < 1e-4
    assert eQ[1] < 0.2 * eQ[0] + 1e-12 and ep[1] < 0.2 * ep[0] + 1e-12
    HX, Hp = native._rtr_joint_hvp(args, X, dp, Q, p, Ft)
    HXr, Hpr = oracle._rtr_joint_hvp(args, X, dp, Q, p, Ft)
    np.testing.assert_allclose(HX, HXr, rtol=0, atol=1e-12 * np.max(np.abs(HXr)))
    np.testing.assert_allclose(Hp, Hpr, rtol=0, atol=1e-12 * np.max(np.abs(Hpr)))
    assert abs(float(np.sum(args["w2d"][..., None] * Hp))) < 1e-10 * np.max(np.abs(Hp))


@pytest.mark.parametrize("case", ["layered8", "dirac16", "refP"])
def test_joint_hvp_larger_meshes(native, oracle, case):
    """nb = 8 (warp teams, small-nb Fock path), nb = 2, and a kernel with a
    reference density (the response must drop it)."""
    rng = np.random.default_rng(5)
    if case == "layered8":
        args, _P0, _ne = workloads.layered(12, seed=1)
    elif case == "dirac16":
        args, _P0, _ne = workloads.dirac(16, seed=3)
    else:
        args, _P0, _ne = workloads.dirac(8, seed=2)
        args = dict(args)
        args["refP"] = herm(rng.standard_normal(args["h"].shape) + 1j * rng.standard_normal(args["h"].shape))
        args["has_refP"] = True
    h = args["h"]
    nb = h.shape[-1]
    eps, Q = np.linalg.eigh(h)
    p = 1.0 / (1.0 + np.exp(eps / 0.1))
    X = rng.standard_normal(h.shape) + 1j * rng.standard_normal(h.shape)
    X = 0.5 * (X - np.conj(np.swapaxes(X, -1, -2)))
    X[..., np.arange(nb), np.arange(nb)] = 0.0
    dp = 0.1 * rng.standard_normal(p.shape)
    Ft = np.conj(np.swapaxes(Q, -1, -2)) @ h @ Q
    HX, Hp = native._rtr_joint_hvp(args, X, dp, Q, p, Ft)
    HXr, Hpr = oracle._rtr_joint_hvp(args, X, dp, Q, p, Ft)
    np.testing.assert_allclose(HX, HXr, rtol=0, atol=1e-12 * np.max(np.abs(HXr)))
    np.testing.assert_allclose(Hp, Hpr, rtol=0, atol=1e-12 * np.max(np.abs(Hpr)))


def test_deflation_bias_matches_oracle(native, oracle):
    rng = np.random.default_rng(0)
    nk, nb = 3, 4
    w2d = np.arange(nk * nk).reshape(nk, nk).astype(np.float64) + 1.0

    def rh(shape):
        return herm(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))

    P = rh((nk, nk, nb, nb))
    targets = np.stack([0.3 * rh((nk, nk, nb, nb)) + P for _ in range(3)])
    for sigma, length in ((0.7, 0.5), (2.0, 3.0)):
        Phi, S, d = native._deflation_bias(P, targets, w2d, sigma, length)
        Phr, Sr, dr = oracle._deflation_bias(P, targets, w2d, sigma, length)
        assert abs(Phi - Phr) <= 1e-13 * max(1.0, abs(Phr))
        assert abs(d - dr) <= 1e-13 * max(1.0, abs(dr))
        np.testing.assert_allclose(S, Sr, rtol=0, atol=1e-13 * max(1.0, np.max(np.abs(Sr))))
    Phi0, S0, d0 = native._deflation_bias(P, np.empty((0, nk, nk, nb, nb), np.complex128), w2d, 1.0, 1.0)
    assert Phi0 == 0.0 and d0 == 0.0 and np.max(np.abs(S0)) == 0.0
    Phi0, S0, d0 = native._deflation_bias(P, targets, w2d, 0.0, 1.0)
    assert Phi0 == 0.0 and d0 == 0.0 and np.max(np.abs(S0)) == 0.0


def _compare(got, ref, tol_E=1e-9, tol_D=1e-7, iters=0):
    print(f"  iterations gpu {got['n_iter']} oracle {ref['n_iter']}, converged {got['converged']}/"
          f"{ref['converged']}, |dE| {abs(got['energy'] - ref['energy']):.2e}")
    assert got["converged"] == ref["converged"]
    assert abs(got["energy"] - ref["energy"]) <= tol_E * max(1.0, abs(ref["energy"]))
    assert np.max(np.abs(got["density"] - ref["density"])) <= tol_D
    assert abs(got["n_iter"] - ref["n_iter"]) <= iters
    # occupations, not mu: inside a gap much wider than T every mu in the gap
    # gives the same occupations to rounding, and the in-loop solve may stop
    # anywhere there (the stiff multiband case has a gap of about 10 at T = 0.015)
    np.testing.assert_allclose(got["p"], ref["p"], rtol=0, atol=1e-7)
    n = min(got["n_iter"], ref["n_iter"])
    np.testing.assert_allclose(got["hist_E"][:n], ref["hist_E"][:n], rtol=1e-9, atol=1e-9)


def _cases():
    out = {}
    out["contact"] = (*nc.contact(g=0.3, nk=2), 4.0, dict(max_iter=200, tol_grad=1e-7))
    args, h = nc.multiband(4, 4, 0.05, 0.3, 7)
    out["multiband4"] = (args, h, 4 * 4 * 4 * 0.5, dict(max_iter=200, tol_grad=1e-6))
    args, h = nc.multiband(6, 6, 0.015, 0.4, 21)
    out["multiband6_stiff"] = (args, h, 6 * 6 * 6 * 0.5, dict(max_iter=200, tol_grad=1e-6))
    out["two_band"] = (*nc.two_band(nk=2, T=0.1), 4.0, dict(max_iter=100, tol_grad=1e-6))
    out["hybridized_projected"] = (*nc.hybridized(nk=2, ex=0.25), 4.0,
                                   dict(max_iter=200, tol_grad=1e-6, project_fn=nc.diag_projector))
    args, P0, ne = workloads.layered(12, seed=1)
    out["layered12_nb8"] = (args, P0, ne, dict(max_iter=100, tol_grad=1e-6))
    out["layered12_delta0.1_cg5"] = (args, P0, ne, dict(max_iter=100, tol_grad=1e-6, tr_delta0=0.1, tr_cg_max=5))
    return out


_CASES = _cases()


@pytest.mark.parametrize("name", sorted(_CASES))
def test_newton_solve_matches_oracle(native, oracle, name):
    args, h, ne, kw = _CASES[name]
    P0 = np.zeros_like(h)
    got = nc.solve(native, args, P0, ne, optimizer="newton", **kw)
    ref = nc.solve(oracle, args, P0, ne, optimizer="newton", **kw)
    print(name)
    _compare(got, ref)
    if ref["converged"]:
        assert nc.comm_rms(got["fock"], got["density"], args["w2d"]) < 1e-4
    if "project_fn" in kw:  # the diagonal projector is enforced (test_deflation.py:57-80)
        assert np.max(np.abs(got["density"][..., 0, 1])) < 1e-8


def test_newton_with_deflation_bias_matches_oracle(native, oracle):
    """A biased solve (target = the converged ground state, sigma > 0): energies
    include the bias, the Hessian gets the bias curvature."""
    args, h = nc.bistable()
    P0 = np.zeros_like(h)
    base = dict(optimizer="newton", tol_grad=1e-6, max_iter=300)
    r0 = nc.solve(oracle, args, P0, 1.0, **base)
    rng = np.random.default_rng(1)
    seed = P0 + 2e-2 * herm(rng.standard_normal(P0.shape) + 1j * rng.standard_normal(P0.shape))
    kw = dict(base, deflation_targets=r0["density"][None], deflation_sigma=3.0, deflation_length=0.5)
    got = nc.solve(native, args, seed, 1.0, **kw)
    ref = nc.solve(oracle, args, seed, 1.0, **kw)
    _compare(got, ref)


def test_deflated_search_matches_oracle(native, oracle):
    args, h = nc.bistable()
    g0, gb, g1, ga = deflated_second_solution(native, args, h)
    r0, rb, r1, ra = deflated_second_solution(oracle, args, h)
    assert ga == ra and ga is not None
    for g, r in ((g0, r0), (gb, rb), (g1, r1)):
        _compare(g, r)
    assert abs(g1["energy"] + 0.4) < 3e-2


def test_newton_deflation_noop_and_errors(native):
    args, h = nc.hybridized(nk=2, ex=0.3)
    P0 = np.zeros_like(h)
    base = dict(optimizer="newton", tol_grad=1e-7, max_iter=200)
    r1 = nc.solve(native, args, P0, 4.0, **base)
    r3 = nc.solve(native, args, P0, 4.0, deflation_targets=r1["density"][None], deflation_sigma=0.0, **base)
    np.testing.assert_array_equal(r3["density"], r1["density"])
    assert r3["energy"] == r1["energy"]
    with pytest.raises(ValueError):
        native.solve_dm(args, P0, 4.0, 10, 1e-7, 1e-6, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 1, 0.5, 20,
                        np.zeros((1, 2, 2, 2, 1), np.complex128), 1.0, 1.0, [], None, True, True, True)
    # any optimizer code other than 1 runs the CG solver (cpp_hf_native.cpp:557-559)
    r_cg = nc.solve(native, args, P0, 4.0, max_iter=50)
    r_2 = native.solve_dm(args, P0, 4.0, 50, 1e-7, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 2, 0.5, 20,
                          np.empty((0, 2, 2, 2, 2), np.complex128), 0.0, 1.0, [], None, True, True, True)
    assert r_2[5] == r_cg["energy"] and r_2[6] == r_cg["n_iter"]


def test_newton_full_size_history_matches_oracle(native):
    """The 192x192, nb = 8 layered workload: the GPU solve against the oracle's
    history (tests/golden/newton_layered192.npz, made by make_oracle_golden.py)."""
    from conftest import GOLDEN

    g = np.load(GOLDEN / "newton_layered192.npz")
    args, P0, ne = workloads.layered(192, seed=0)
    r = nc.solve(native, args, P0, ne, optimizer="newton", tol_grad=1e-6, max_iter=60)
    print(f"  newton 192^2: iterations gpu {r['n_iter']} oracle {int(g['n_iter'])}, "
          f"|dE| {abs(r['energy'] - float(g['energy'])):.2e}")
    assert r["n_iter"] == int(g["n_iter"]) and r["converged"] == bool(g["converged"])
    assert abs(r["energy"] - float(g["energy"])) < 1e-10 * abs(float(g["energy"]))
    np.testing.assert_allclose(r["hist_E"], g["hist_E"], rtol=1e-11, atol=0)
    np.testing.assert_allclose(r["hist_grad"], g["hist_grad"], rtol=1e-7, atol=0)
    assert abs(float(np.sum(r["p"])) - float(g["p_sum"])) < 1e-8 * abs(float(g["p_sum"]))
