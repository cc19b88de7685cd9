"""Write oracle outputs too slow to recompute inside the GPU tests.

``newton_layered192.npz``: the trust-region Newton solve (optimizer=1) of the
192x192, nb = 8 layered workload (seed 0, tol_grad 1e-6, max_iter 60) by
``oracle.native_np`` (about three minutes on one core): the energy and
gradient-norm histories, the final energy, the iteration count and the sum of
the occupations.

Usage: ``python tests/golden/make_oracle_golden.py``
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

import newton_cases as nc  # noqa: E402
from cpp_hf_b200 import workloads  # noqa: E402
from oracle import native_np  # noqa: E402

NEWTON_192 = dict(n=192, seed=0, tol_grad=1e-6, max_iter=60)
DIRAC_48 = dict(n=48, seed=0, tol_E=1e-10, max_iter=200)
LAYERED_192 = dict(n=192, seed=0, tol_E=1e-10, max_iter=1000, scf_tol=1e-9, mixing=0.5, n_probe=64)


def dm_call(mod, args, P0, n_e, tol_E, max_iter):
    """solve() with cpp_hf's SolverConfig defaults except tol_E / max_iter (solver.py:19-64)."""
    nk1, nk2, nb = P0.shape[0], P0.shape[1], P0.shape[2]
    defl = np.empty((0, nk1, nk2, nb, nb), np.complex128)
    return mod.solve_dm(args, P0, n_e, max_iter, tol_E, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, defl, 0.0,
                        1.0, [], None, True, True, True)


def scf_call(mod, args, P0, n_e, tol, mixing, max_iter):
    """solve_scf with linear mixing and equal density / commutator tolerances."""
    return mod.solve_scf(args, P0, n_e, max_iter, tol, tol, mixing, 0.0, None, [], "linear", 6, 2, 1.0, 0.0,
                         True, True)


def probe_index(n, count, seed=1234):
    """Seeded k-points (flat indices) at which full matrices are stored."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n * n, size=count, replace=False))


def field_checksums(X, w, idx):
    """(sum_k w_k X(k), sum_k w_k |X(k)|_F^2, X at the probe k-points) of an (n, n, nb, nb) field."""
    nb = X.shape[-1]
    flat = X.reshape(-1, nb, nb)
    wf = np.asarray(w, np.float64).reshape(-1)
    return (np.einsum("k,kij->ij", wf, flat), np.float64(np.sum(wf * np.sum(np.abs(flat) ** 2, axis=(1, 2)))),
            flat[idx].copy())


def dm_dirac48():
    c = DIRAC_48
    args, P0, ne = workloads.dirac(c["n"], seed=c["seed"])
    Q, p, D, F, mu, E, it, conv, hE, hG = dm_call(native_np, args, P0, ne, c["tol_E"], c["max_iter"])
    np.savez_compressed(HERE / "dm_dirac48.npz", hist_E=hE, hist_grad=hG, energy=np.float64(E), mu=np.float64(mu),
                        n_iter=np.int64(it), converged=np.bool_(conv), p=p, density=D, fock=F)


def dm_layered192():
    c = LAYERED_192
    args, P0, ne = workloads.layered(c["n"], seed=c["seed"])
    idx = probe_index(c["n"], c["n_probe"])
    Q, p, D, F, mu, E, it, conv, hE, hG = dm_call(native_np, args, P0, ne, c["tol_E"], c["max_iter"])
    Dw, Dn, Dp = field_checksums(D, args["w2d"], idx)
    Fw, Fn, Fp = field_checksums(F, args["w2d"], idx)
    np.savez_compressed(HERE / "dm_layered192.npz", hist_E=hE, hist_grad=hG, energy=np.float64(E),
                        mu=np.float64(mu), n_iter=np.int64(it), converged=np.bool_(conv), p_sum=np.float64(np.sum(p)),
                        probe=idx, D_wsum=Dw, D_wnorm=Dn, D_probe=Dp, F_wsum=Fw, F_wnorm=Fn, F_probe=Fp)


def scf_layered192():
    c = LAYERED_192
    args, P0, ne = workloads.layered(c["n"], seed=c["seed"])
    idx = probe_index(c["n"], c["n_probe"])
    D, F, E, mu, it, conv, hE, hD, hC = scf_call(native_np, args, P0, ne, c["scf_tol"], c["mixing"], c["max_iter"])
    Dw, Dn, Dp = field_checksums(D, args["w2d"], idx)
    Fw, Fn, Fp = field_checksums(F, args["w2d"], idx)
    np.savez_compressed(HERE / "scf_layered192.npz", hist_E=hE, hist_D=hD, hist_C=hC, energy=np.float64(E),
                        mu=np.float64(mu), n_iter=np.int64(it), converged=np.bool_(conv),
                        probe=idx, D_wsum=Dw, D_wnorm=Dn, D_probe=Dp, F_wsum=Fw, F_wnorm=Fn, F_probe=Fp)


def newton_layered192():
    c = NEWTON_192
    args, P0, ne = workloads.layered(c["n"], seed=c["seed"])
    r = nc.solve(native_np, args, P0, ne, optimizer="newton", tol_grad=c["tol_grad"], max_iter=c["max_iter"])
    np.savez_compressed(HERE / "newton_layered192.npz", hist_E=r["hist_E"], hist_grad=r["hist_grad"],
                        energy=np.float64(r["energy"]), mu=np.float64(r["mu"]), n_iter=np.int64(r["n_iter"]),
                        converged=np.bool_(r["converged"]), p_sum=np.float64(np.sum(r["p"])))


MAKERS = {"newton_layered192": newton_layered192, "dm_dirac48": dm_dirac48, "dm_layered192": dm_layered192,
          "scf_layered192": scf_layered192}

if __name__ == "__main__":
    for name in (sys.argv[1:] or list(MAKERS)):
        MAKERS[name]()
