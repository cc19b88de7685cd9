"""CPU: pin the oracle and the kernel-argument precompute against reference data.

* ``meshgrid_scf_v1.npz``: the reference's stored SCF regression case
  (``tests/data/meshgrid_regression_case_v1.npz``), checked at 1e-6 like
  ``examples/contimod_example_meshgrid_offline.py:84-94``.
* ``kernel_args_ref.npz``: kernel_args dicts produced by the reference's own
  ``HartreeFockKernel`` (``src/cpp_hf/problem.py:24-228``).
* Analytic identities the reference tests rely on (``tests/test_main.py:43-48``,
  ``tests/test_solver.py:280-347``, ``tests/test_linalg.py:75-94``).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, herm, rand_herm
from cpp_hf_b200 import problem, workloads
from oracle import native_np as nn


def _mesh_case():
    d = np.load(GOLDEN / "meshgrid_scf_v1.npz")
    args = problem.kernel_args(d["weights"], d["hamiltonian"], d["coulomb_q"], float(d["T"]),
                               include_hartree=True, include_exchange=True,
                               reference_density=d["reference_density"],
                               hartree_matrix=d["hartree_matrix"])
    return d, args


def test_meshgrid_regression_case_matches_stored_results():
    d, args = _mesh_case()
    out = nn.solve_scf(args, np.asarray(d["P0"]), float(d["electrondensity0"]), int(d["max_iter"]),
                       float(d["comm_tol"]), float(d["comm_tol"]), 0.5, 0.0, None, [], "linear", 6, 2,
                       1.0, 0.0, True, True)
    density, fock, energy, mu, iters, conv = out[:6]
    hist_C = out[8]
    assert conv
    np.testing.assert_allclose(density, d["P_expected"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(fock, d["F_expected"], rtol=1e-6, atol=1e-6)
    assert abs(mu - float(d["mu_expected"])) < 1e-6
    # first-iteration commutator residual (independent of the v1 acceleration)
    assert abs(hist_C[0] - float(d["hist_dC_expected"][0])) < 1e-6
    # energy in the v1 convention Re Tr[h P + (Sigma + H) P / 2]
    S, H, _F, _E = nn.build_fock_apply(args, d["P_expected"].astype(np.complex128), None)
    w = args["w2d"]
    tr = lambda A, B: float(np.sum(w * np.real(np.einsum("...ij,...ji->...", A, B))))  # noqa: E731
    E_v1 = tr(args["h"], d["P_expected"]) + 0.5 * tr(S + H, d["P_expected"])
    assert abs(E_v1 - float(d["E_expected"])) < 1e-6


@pytest.mark.parametrize("name", ["scalar", "layered"])
def test_kernel_args_match_reference_hartree_fock_kernel(name):
    g = np.load(GOLDEN / "kernel_args_ref.npz")
    kw = dict(T=float(g[f"{name}.in.T"]))
    if f"{name}.in.include_hartree" in g.files:
        kw.update(include_hartree=bool(g[f"{name}.in.include_hartree"]),
                  reference_density=g[f"{name}.in.reference_density"],
                  hartree_matrix=g[f"{name}.in.hartree_matrix"])
    if f"{name}.in.contact_g" in g.files:
        kw["contact_terms"] = list(zip(g[f"{name}.in.contact_g"], g[f"{name}.in.contact_Oi"],
                                       g[f"{name}.in.contact_Oj"]))
    args = problem.kernel_args(g[f"{name}.in.weights"], g[f"{name}.in.hamiltonian"],
                               g[f"{name}.in.coulomb_q"], **kw)
    for key in ["h", "VR", "refP", "w2d", "HH", "contact_g", "contact_Oi", "contact_Oj"]:
        np.testing.assert_allclose(args[key], g[f"{name}.out.{key}"], rtol=1e-13, atol=1e-13,
                                   err_msg=key)
    for key in ["has_refP", "include_hartree", "include_exchange", "exchange_hcp"]:
        assert bool(args[key]) == bool(g[f"{name}.out.{key}"]), key
    assert abs(args["weight_sum"] - float(g[f"{name}.out.weight_sum"])) < 1e-13
    assert abs(args["T"] - float(g[f"{name}.out.T"])) < 1e-15


def test_single_point_exchange_is_minus_v_times_p():
    VR = np.array([[[[0.3]]]], dtype=np.complex128)
    P = np.array([[[[1.0 + 0.5j, 0.2], [0.2, 0.8 - 0.1j]]]])
    np.testing.assert_allclose(nn.selfenergy_fft_full(VR, P), -VR * P, rtol=1e-15, atol=1e-15)


def test_hcp_matches_full_for_hermitian_density():
    rng = np.random.default_rng(3)
    P = rand_herm(rng, (6, 5, 3, 3))
    # a real scalar interaction (the HCP precondition, problem.py:92-94)
    Vq = rng.normal(size=(6, 5, 1, 1))
    VR = np.fft.fftn(Vq / 30.0, axes=(0, 1)) * problem.shift_phase(6, 5)[..., None, None]
    a = nn.selfenergy_fft_full(VR, P, False, False)
    b = nn.selfenergy_fft_full(VR, P, False, True)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_spectral_cayley_matches_lu_cayley():
    rng = np.random.default_rng(0)
    d = rng.normal(size=(3, 3, 6, 6)) + 1j * rng.normal(size=(3, 3, 6, 6))
    d = 0.5 * (d - np.conj(np.swapaxes(d, -1, -2)))
    V, lam = nn._cayley_spectral_setup(d)
    eye = np.eye(6)
    for tau in [0.0, 0.1, 0.5, -0.3]:
        A = 0.5 * tau * d
        U_lu = np.linalg.solve(eye + A, eye - A)
        np.testing.assert_allclose(nn._cayley_unitary_from_spectrum(V, lam, tau), U_lu, atol=1e-12)


def test_dirac_workload_solves_and_is_self_consistent():
    args, P0, n_e = workloads.dirac(8, seed=1)
    out = nn.solve_dm(args, P0, n_e, 200, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                      np.empty((0, 8, 8, 2, 2), np.complex128), 0.0, 1.0, [], None, True, True, True)
    Q, p, D, F = out[:4]
    assert out[7]
    comm = F @ D - D @ F
    assert np.sqrt(np.sum(args["w2d"] * np.sum(np.abs(comm) ** 2, axis=(-2, -1)))) < 1e-4
    assert abs(np.sum(args["w2d"][..., None] * p) - n_e) < 1e-8


def test_layered_workload_shapes_and_symmetry():
    args, P0, n_e = workloads.layered(6, n_layers=2, seed=2)
    assert args["VR"].shape == (6, 6, 4, 4)
    assert not args["exchange_hcp"]
    np.testing.assert_allclose(args["h"], herm(args["h"]), atol=1e-15)
    assert abs(n_e - 2.0) < 1e-12


def test_superlattice_layout_and_kernel_args_match_reference_fixture():
    """cpp_hf_b200.superlattice against the reference's build_extended_layout +
    SuperlatticeHartreeFockKernel (tests/golden/superlattice_ref.npz)."""
    from cpp_hf_b200 import superlattice as sl

    d = np.load(GOLDEN / "superlattice_ref.npz")
    n = int(d["in.n"])
    V = lambda q: 2 * np.pi * 0.5 / (q + 0.05) * np.tanh(5 * q)  # noqa: E731
    lay = sl.extended_layout(d["in.g_frac"], d["in.B"], n, n, V, float(d["in.w_scalar"]))
    args = sl.superlattice_kernel_args(np.full((n, n), 1.0 / n ** 2), d["in.h"], lay, 0.05, HH_GG=d["in.HH_GG"],
                                       hartree_degeneracy=2.0)
    for key in d.files:
        if not key.startswith("out."):
            continue
        k = key[4:]
        ref = d[key]
        got = np.asarray(args[k])
        if ref.size == 0 and got.size == 0:
            continue
        if k == "refP":  # the reference passes an empty refP without a reference density
            assert not args["has_refP"] and ref.size == 0
            continue
        assert got.shape == ref.shape, k
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13, err_msg=k)


def _symmetry_kwargs(G, S, U):
    """The projector configurations of tests/golden/make_golden.py:_symmetry_cases."""
    return {
        "unitary": dict(unitary_group=G),
        "spatial_mod": dict(spatial_group=S),
        "spatial_flip_axis0": dict(spatial_group=S, spatial_k_convention="flip", spatial_k_flip_axes=(0,)),
        "combined": dict(unitary_group=G, spatial_group=S),
        "tr_mod": dict(time_reversal_U=U),
        "tr_flip_axis1": dict(time_reversal_U=U, time_reversal_k_convention="flip", time_reversal_k_flip_axes=(1,)),
        "all": dict(unitary_group=G, spatial_group=S, time_reversal_U=U, spatial_k_flip_axes=(1,)),
    }


def test_symmetry_projector_restatement_matches_reference_vectors():
    """oracle/symmetry_np.py against outputs of the reference's
    cpp_hf.symmetry.make_project_fn (tests/golden/symmetry_ref.npz)."""
    from oracle import symmetry_np

    d = np.load(GOLDEN / "symmetry_ref.npz")
    for name, kw in _symmetry_kwargs(d["in.G"], d["in.S"], d["in.U"]).items():
        got = symmetry_np.make_project_fn(**kw)(d["in.A"])
        np.testing.assert_allclose(got, d[f"{name}.out"], rtol=0, atol=1e-14, err_msg=name)
