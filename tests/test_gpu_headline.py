"""GPU: the headline solves against cached FP64 oracle runs at their full sizes.

Fixtures (``tests/golden/make_oracle_golden.py``, oracle = the NumPy FP64
restatement of the reference's solver_dm.hpp / solver_scf.hpp loops):

* ``dm_dirac48.npz``: solve() of the 48 x 48 massive Dirac model (nb = 2,
  scalar V, exchange only, tol_E = 1e-10);
* ``dm_layered192.npz``: solve() of the 192 x 192, nb = 8 layered model
  (layer-resolved V, tol_E = 1e-10);
* ``scf_layered192.npz``: solve_scf() of the same model (linear mixing 0.5,
  density_tol = comm_tol = 1e-9).

Bars: the FP64 GPU solve takes the oracle's iteration count, its energy
history matches step by step, and its converged energy, density and Fock
matrix match within the tolerances below (relative to the largest entry).
The switched-precision solve (complex64 exchange until the residual falls
below 1e-5) must reach the oracle's converged FP64 energy within 1e-9
relative.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN
from cpp_hf_b200 import workloads

pytestmark = pytest.mark.gpu

E_TOL = 1e-9          # converged energies (FP64 and switched precision) vs the FP64 oracle
HIST_TOL = 1e-10      # per-iteration energies of the FP64 solve
FIELD_TOL = 1e-9      # converged density / Fock of the FP64 solve (relative to their largest entry)


def dm_call(native, args, P0, n_e, tol_E, max_iter):
    nk1, nk2, nb = P0.shape[0], P0.shape[1], P0.shape[2]
    defl = np.empty((0, nk1, nk2, nb, nb), np.complex128)
    return native.solve_dm(args, P0, n_e, max_iter, tol_E, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, defl,
                           0.0, 1.0, [], None, True, True, True)


def scf_call(native, args, P0, n_e, tol, mixing, max_iter):
    return native.solve_scf(args, P0, n_e, max_iter, tol, tol, mixing, 0.0, None, [], "linear", 6, 2, 1.0, 0.0,
                            True, True)


def rel_field(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def checksums(X, w, idx):
    nb = X.shape[-1]
    flat = X.reshape(-1, nb, nb)
    wf = np.asarray(w, np.float64).reshape(-1)
    return (np.einsum("k,kij->ij", wf, flat), float(np.sum(wf * np.sum(np.abs(flat) ** 2, axis=(1, 2)))),
            flat[idx])


def check_fields(g, D, F, w):
    for name, X in (("D", D), ("F", F)):
        ws, wn, probe = checksums(X, w, g["probe"])
        assert rel_field(ws, g[f"{name}_wsum"]) < FIELD_TOL, name
        assert abs(wn - float(g[f"{name}_wnorm"])) < FIELD_TOL * float(g[f"{name}_wnorm"]), name
        assert rel_field(probe, g[f"{name}_probe"]) < FIELD_TOL, name


@pytest.fixture(scope="module")
def layered192():
    return workloads.layered(192, n_layers=4, seed=0)


def test_dm_dirac48_fp64_matches_oracle(native):
    g = np.load(GOLDEN / "dm_dirac48.npz")
    args, P0, n_e = workloads.dirac(48, seed=0)
    Q, p, D, F, mu, E, it, conv, hE, hG = dm_call(native, args, P0, n_e, 1e-10, 200)
    assert conv and bool(g["converged"])
    assert it == int(g["n_iter"])
    assert np.max(np.abs(hE - g["hist_E"])) < HIST_TOL * abs(float(g["energy"]))
    assert abs(E - float(g["energy"])) < E_TOL * abs(float(g["energy"]))
    assert rel_field(D, g["density"]) < FIELD_TOL
    assert rel_field(F, g["fock"]) < FIELD_TOL
    assert float(np.max(np.abs(p - g["p"]))) < FIELD_TOL


def test_dm_dirac48_mixed_reaches_oracle_energy(native):
    g = np.load(GOLDEN / "dm_dirac48.npz")
    args, P0, n_e = workloads.dirac(48, seed=0)
    args = dict(args, exchange_precision="mixed")
    r = dm_call(native, args, P0, n_e, 1e-10, 200)
    assert r[7]
    assert abs(r[5] - float(g["energy"])) < E_TOL * abs(float(g["energy"]))


def test_dm_layered192_fp64_matches_oracle(native, layered192):
    g = np.load(GOLDEN / "dm_layered192.npz")
    args, P0, n_e = layered192
    Q, p, D, F, mu, E, it, conv, hE, hG = dm_call(native, args, P0, n_e, 1e-10, 1000)
    assert conv and bool(g["converged"])
    assert it == int(g["n_iter"])
    assert np.max(np.abs(hE - g["hist_E"])) < HIST_TOL * abs(float(g["energy"]))
    assert abs(E - float(g["energy"])) < E_TOL * abs(float(g["energy"]))
    assert abs(float(np.sum(p)) - float(g["p_sum"])) < 1e-9 * float(g["p_sum"])
    check_fields(g, D, F, args["w2d"])


def test_dm_layered192_mixed_reaches_oracle_energy(native, layered192):
    g = np.load(GOLDEN / "dm_layered192.npz")
    args, P0, n_e = layered192
    r = dm_call(native, dict(args, exchange_precision="mixed"), P0, n_e, 1e-10, 1000)
    assert r[7]
    assert abs(r[5] - float(g["energy"])) < E_TOL * abs(float(g["energy"]))


def test_scf_layered192_fp64_matches_oracle(native, layered192):
    g = np.load(GOLDEN / "scf_layered192.npz")
    args, P0, n_e = layered192
    D, F, E, mu, it, conv, hE, hD, hC = scf_call(native, args, P0, n_e, 1e-9, 0.5, 1000)
    assert conv and bool(g["converged"])
    assert it == int(g["n_iter"])
    assert np.max(np.abs(hE - g["hist_E"])) < HIST_TOL * abs(float(g["energy"]))
    assert abs(E - float(g["energy"])) < E_TOL * abs(float(g["energy"]))
    check_fields(g, D, F, args["w2d"])


def test_scf_layered192_mixed_reaches_oracle_energy(native, layered192):
    g = np.load(GOLDEN / "scf_layered192.npz")
    args, P0, n_e = layered192
    r = scf_call(native, dict(args, exchange_precision="mixed"), P0, n_e, 1e-9, 0.5, 1000)
    assert r[5]
    assert abs(r[2] - float(g["energy"])) < E_TOL * abs(float(g["energy"]))
