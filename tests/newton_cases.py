"""Problems and a call helper for the trust-region Newton tests (CPU and GPU).

The kernels follow the shapes and parameters of the reference's Newton and
deflation tests (``tests/test_solver_rtr.py:27-69``, ``tests/test_deflation.py:24-53``):
a two-band model, a two-band contact model with a unique HF minimum, a random
multiband model, a hybridised two-band model and a bistable one-k-point model.
"""

from __future__ import annotations

import numpy as np

from cpp_hf_b200 import problem

# SolverConfig defaults (src/cpp_hf/solver.py:29-59)
DEFAULTS = dict(max_iter=200, tol_E=1e-7, tol_grad=0.0, max_step=0.6, bt_shrink=0.5, denom_scale=1e-3, bt_max=8,
                cg_restart=10, plateau_window=5, mu_maxiter=25, optimizer="cg", tr_delta0=0.5, tr_cg_max=20,
                deflation_targets=None, deflation_sigma=0.0, deflation_length=1.0, block_sizes=(),
                project_fn=None)


def solve(mod, args, P0, n_e, **kw):
    """``_native.solve_dm`` called the way ``solver.solve_direct_minimization`` calls it
    (src/cpp_hf/solver.py:150-226); returns the binding's 10-tuple as a dict."""
    c = dict(DEFAULTS)
    c.update(kw)
    nk1, nk2, nb = P0.shape[0], P0.shape[1], P0.shape[-1]
    t = c["deflation_targets"]
    if t is None:
        t = np.empty((0, nk1, nk2, nb, nb), np.complex128)
    t = np.ascontiguousarray(t, np.complex128)
    if t.ndim == 4:
        t = t[None]
    out = mod.solve_dm(args, np.ascontiguousarray(P0, np.complex128), float(n_e), int(c["max_iter"]),
                       float(c["tol_E"]), float(c["tol_grad"]), float(c["max_step"]), float(c["bt_shrink"]),
                       float(c["denom_scale"]), int(c["bt_max"]), int(c["cg_restart"]), int(c["plateau_window"]),
                       int(c["mu_maxiter"]), {"cg": 0, "newton": 1}[c["optimizer"]], float(c["tr_delta0"]),
                       int(c["tr_cg_max"]), t, float(c["deflation_sigma"]), float(c["deflation_length"]),
                       list(c["block_sizes"]), c["project_fn"], True, True, True)
    keys = ("Q", "p", "density", "fock", "mu", "energy", "n_iter", "converged", "hist_E", "hist_grad")
    return dict(zip(keys, out))


def comm_rms(F, P, w2d):
    c = F @ P - P @ F
    per_k = np.sum(np.abs(c) ** 2, axis=(-2, -1))
    return float(np.sqrt(np.sum(w2d * per_k) / max(float(np.sum(w2d)), 1e-30)))


def _args(w, h, vq, T, **kw):
    return problem.kernel_args(w, h.astype(np.complex128), vq, T, **kw)


def two_band(nk=2, T=0.1, ex=0.25):
    w = np.ones((nk, nk))
    h = np.zeros((nk, nk, 2, 2), np.complex128)
    h[..., 0, 0], h[..., 1, 1] = -0.5, 0.5
    return _args(w, h, np.full((nk, nk, 1, 1), ex, np.complex128), T), h


def contact(g=0.3, nk=2, T=0.05):
    w = np.ones((nk, nk))
    h = np.zeros((nk, nk, 2, 2), np.complex128)
    h[..., 0, 0], h[..., 1, 1] = -1.0, 1.0
    for i in range(nk):
        for j in range(nk):
            h[i, j, 0, 1] = h[i, j, 1, 0] = 0.4 + 0.1 * (i + j)
    sz = np.diag([1.0, -1.0]).astype(np.complex128)
    return _args(w, h, np.full((nk, nk, 1, 1), 0.1, np.complex128), T,
                 contact_terms=[(g, sz, sz)]), h


def multiband(nk, nb, T, ex, seed):
    rng = np.random.default_rng(seed)
    w = np.ones((nk, nk))
    A = (rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))) * 0.35
    A = 0.5 * (A + A.conj().T)
    kx = np.arange(nk) / nk * 2 * np.pi
    h = np.zeros((nk, nk, nb, nb), np.complex128)
    for i in range(nk):
        for j in range(nk):
            hk = np.diag(np.linspace(-1.0, 1.0, nb)).astype(np.complex128) + A * (np.cos(kx[i]) + np.cos(kx[j]))
            h[i, j] = 0.5 * (hk + hk.conj().T)
    # the reference builds these kernels from complex64 arrays
    h = h.astype(np.complex64).astype(np.complex128)
    return _args(w, h, np.full((nk, nk, 1, 1), ex, np.complex128), T), h


def hybridized(nk=2, T=0.05, ex=0.25):
    w = np.ones((nk, nk))
    h = np.zeros((nk, nk, 2, 2), np.complex128)
    h[..., 0, 0], h[..., 1, 1] = -0.5, 0.5
    h[..., 0, 1] = h[..., 1, 0] = 0.3
    return _args(w, h, np.full((nk, nk, 1, 1), ex, np.complex128), T), h


def bistable(nk=1, T=0.02, ex=1.0, delta=0.1):
    """Two self-consistent solutions: diag(1, 0) at E = -delta - ex/2 and diag(0, 1)
    at E = +delta - ex/2."""
    w = np.ones((nk, nk))
    h = np.zeros((nk, nk, 2, 2), np.complex128)
    h[..., 0, 0], h[..., 1, 1] = -delta, delta
    return _args(w, h, np.full((nk, nk, 1, 1), ex, np.complex128), T), h


def diag_projector(P):
    P = np.array(P, copy=True)
    P[..., 0, 1] = 0.0
    P[..., 1, 0] = 0.0
    return P
