"""GPU: superlattice (moire plane-wave) Fock terms against the oracle -- the
streamed Delta-G exchange (selfenergy_superlattice_streamed), the superlattice
Hartree, Fock builds and solves through superlattice kernel_args, and the
nb = 64 Dirac superlattice at a small mesh."""

from __future__ import annotations

import numpy as np
import pytest

from cpp_hf_b200 import superlattice as sl

pytestmark = pytest.mark.gpu

V = lambda q: 2 * np.pi * 0.5 / (q + 0.05) * np.tanh(5 * q)  # noqa: E731


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _layout(n_pw=7, n=6):
    g, B = sl._triangular_shells(n_pw)
    return g, sl.extended_layout(g, B, n, n, V, 1.0 / n ** 2)


def _rho(rng, n, nG, orb, herm):
    D = nG * orb
    r = rng.normal(size=(n, n, D, D)) + 1j * rng.normal(size=(n, n, D, D))
    if herm:
        r = 0.5 * (r + np.conj(np.swapaxes(r, -1, -2)))
    return r.reshape(n, n, nG, orb, nG, orb)


def _call(mod, rho, lay, n, nG, orb, vo=None, herm=False):
    return mod.selfenergy_superlattice_streamed(rho, lay.V_lag_fft, lay.g_a_off, lay.delta_pair_i, lay.delta_pair_j,
                                                lay.delta_pair_start, n, n, nG, orb, lay.N_ext_x, lay.N_ext_y,
                                                VR_fft_orbital=vo, hermitian_rho=herm)


@pytest.mark.parametrize("orb,herm", [(2, False), (2, True), (1, False), (3, True)])
def test_streamed_exchange_matches_oracle(native, oracle, orb, herm):
    n = 6
    g, lay = _layout(7, n)
    rng = np.random.default_rng(orb * 10 + herm)
    rho = _rho(rng, n, g.shape[0], orb, herm)
    got = _call(native, rho, lay, n, g.shape[0], orb, herm=herm)
    ref = _call(oracle, rho, lay, n, g.shape[0], orb, herm=herm)
    assert _rel(got, ref) < 1e-12


def test_streamed_exchange_orbital_coulomb_matches_oracle(native, oracle):
    n, orb = 6, 2
    g, lay = _layout(7, n)
    rng = np.random.default_rng(3)
    vo = (rng.normal(size=(lay.N_ext_x, lay.N_ext_y, orb, orb)) + 1j * rng.normal(size=(lay.N_ext_x, lay.N_ext_y,
                                                                                       orb, orb)))
    rho = _rho(rng, n, g.shape[0], orb, True)
    got = _call(native, rho, lay, n, g.shape[0], orb, vo=vo, herm=True)
    ref = _call(oracle, rho, lay, n, g.shape[0], orb, vo=vo, herm=True)
    assert _rel(got, ref) < 1e-12


def test_streamed_exchange_validation(native):
    n, orb = 6, 2
    g, lay = _layout(7, n)
    rho = np.zeros((n, n, g.shape[0], orb, g.shape[0], orb), np.complex128)
    with pytest.raises(ValueError, match="g_a_off"):
        native.selfenergy_superlattice_streamed(rho, lay.V_lag_fft, lay.g_a_off[:3], lay.delta_pair_i,
                                                lay.delta_pair_j, lay.delta_pair_start, n, n, g.shape[0], orb,
                                                lay.N_ext_x, lay.N_ext_y)
    with pytest.raises(ValueError, match="VR_fft shape"):
        native.selfenergy_superlattice_streamed(rho, lay.V_lag_fft[:5], lay.g_a_off, lay.delta_pair_i,
                                                lay.delta_pair_j, lay.delta_pair_start, n, n, g.shape[0], orb,
                                                lay.N_ext_x, lay.N_ext_y)


def _sl_args(rng, n=6, n_pw=7, orb=2, hartree=True, refP=False, orbital=False):
    g, lay = _layout(n_pw, n)
    nG = g.shape[0]
    D = nG * orb
    h = rng.normal(size=(n, n, D, D)) + 1j * rng.normal(size=(n, n, D, D))
    h = 0.5 * (h + np.conj(np.swapaxes(h, -1, -2)))
    HH = rng.uniform(0.0, 1.0, size=(nG, nG))
    HH = 0.5 * (HH + HH.T)
    np.fill_diagonal(HH, 0.0)
    kw = {}
    if orbital:
        kw["HH_GG_orbital"] = rng.uniform(0.0, 0.5, size=(nG, nG, orb, orb))
        vo = rng.normal(size=(lay.N_ext_x, lay.N_ext_y, orb, orb)) + 0j
        kw["V_lag_fft_orbital"] = vo
    ref = None
    if refP:
        ref = 0.05 * (rng.normal(size=(n, n, D, D)) + 0j)
        ref = 0.5 * (ref + np.conj(np.swapaxes(ref, -1, -2)))
    args = sl.superlattice_kernel_args(np.full((n, n), 1.0 / n ** 2), h, lay, 0.05, HH_GG=HH, include_hartree=hartree,
                                       reference_density=ref, hartree_degeneracy=2.0, **kw)
    return args, D


@pytest.mark.parametrize("hartree,refP,orbital", [(True, False, False), (True, True, False), (False, False, False),
                                                  (True, False, True)])
def test_build_fock_superlattice_matches_oracle(native, oracle, hartree, refP, orbital):
    rng = np.random.default_rng(7)
    args, D = _sl_args(rng, hartree=hartree, refP=refP, orbital=orbital)
    n = args["h"].shape[0]
    P = rng.normal(size=(n, n, D, D)) + 1j * rng.normal(size=(n, n, D, D))
    P = 0.5 * (P + np.conj(np.swapaxes(P, -1, -2)))
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert _rel(S, Sr) < 1e-12
    assert _rel(F, Fr) < 1e-12
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er))


@pytest.mark.parametrize("hartree", [False, True])
def test_solve_superlattice_matches_oracle(native, oracle, hartree):
    """Direct minimisation through superlattice kernel_args (streamed exchange, and
    the superlattice Hartree) converges to the oracle's energy on the Dirac
    superlattice (7 plane waves x 2, 6 x 6 mesh)."""
    a2, P0, n_e = sl.dirac_superlattice(6, n_pw=7, seed=2, hartree=hartree)
    D = P0.shape[-1]
    empty = np.empty((0, 6, 6, D, D), np.complex128)
    got = native.solve_dm(a2, P0, n_e, 500, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0, 1.0,
                          [], None, False, True, False)
    ref = oracle.solve_dm(a2, P0, n_e, 500, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0, 1.0,
                          [], None, False, True, False)
    print(f"Dirac superlattice DM (hartree={hartree}): iterations gpu {got[6]} oracle {ref[6]}, "
          f"|dE| {abs(got[5] - ref[5]):.2e}")
    assert got[7] and ref[7]
    assert abs(got[5] - ref[5]) < 1e-9 * max(1.0, abs(ref[5]))
    assert _rel(got[2], ref[2]) < 1e-6


def test_dirac_superlattice_nb64_build_matches_oracle(native, oracle):
    """The nb = 64 Dirac superlattice (32 plane waves x 2) at a 6 x 6 mesh, streamed
    form; and its plain-mesh form (Hermitian channel packing, 2080 channels)."""
    args, P0, n_e = sl.dirac_superlattice(6, n_pw=32, seed=0)
    rng = np.random.default_rng(1)
    n, D = 6, 64
    A = rng.normal(size=(n, n, D, D)) + 1j * rng.normal(size=(n, n, D, D))
    Q, _ = np.linalg.qr(A)
    P = (Q * rng.uniform(0, 1, size=(n, n, D))[..., None, :]) @ np.conj(np.swapaxes(Q, -1, -2))
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert _rel(S, Sr) < 1e-12 and _rel(F, Fr) < 1e-12
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er))
    a2, _, _ = sl.dirac_superlattice(6, n_pw=32, seed=0, streamed=False)
    assert a2["exchange_hcp"]
    S2, _, F2, E2 = native.build_fock_apply(a2, P, None)
    S2r, _, F2r, E2r = oracle.build_fock_apply(a2, P, None)
    assert _rel(S2, S2r) < 1e-12 and _rel(F2, F2r) < 1e-12


def test_dirac_superlattice_nb64_plain_mesh_solve_matches_oracle(native, oracle):
    """nb = 64 direct minimisation (the plain-mesh form: 32 plane waves x 2, scalar V,
    Hermitian channel packing) on a 6 x 6 mesh against the oracle: the per-k nb = 64
    kernels (Jacobi eigh, elimination Cayley factor, products) of the large-nb path."""
    a2, P0, n_e = sl.dirac_superlattice(6, n_pw=32, seed=0, streamed=False)
    empty = np.empty((0, 6, 6, 64, 64), np.complex128)
    call = (a2, P0, n_e, 300, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0, 1.0, [], None,
            False, True, True)
    got = native.solve_dm(*call)
    ref = oracle.solve_dm(*call)
    assert got[7] and ref[7]
    assert got[6] == ref[6]
    assert abs(got[5] - ref[5]) < 1e-9 * max(1.0, abs(ref[5]))
    assert _rel(got[2], ref[2]) < 1e-8
