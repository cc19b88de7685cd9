"""GPU parity: every ``_native`` entry point of the CUDA library against the oracle.

Small seeded inputs the oracle finishes in seconds; tolerances follow the
reference's own tests (``tests/test_main.py``, ``tests/test_solver.py``,
``tests/test_linalg.py``) and the FP64 parity bar (fields 1e-10 relative,
exchange 1e-12).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import herm, rand_herm
from cpp_hf_b200 import problem, workloads

pytestmark = pytest.mark.gpu

EMPTY_DEFL = None


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _scalar_VR(rng, n0, n1):
    Vq = np.abs(rng.normal(size=(n0, n1, 1, 1))) + 0.1
    return np.fft.fftn(Vq / (n0 * n1), axes=(0, 1)) * problem.shift_phase(n0, n1)[..., None, None]


# ---------------------------------------------------------------------------
# exchange
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n0,n1,nb", [(1, 1, 1), (1, 1, 2), (2, 3, 2), (12, 12, 4), (5, 7, 3),
                                      (48, 48, 2), (36, 72, 3), (11, 13, 2), (96, 96, 8), (144, 48, 2)])
@pytest.mark.parametrize("shift", [False, True])
def test_exchange_full_elementwise(native, oracle, n0, n1, nb, shift):
    rng = np.random.default_rng(n0 * 100 + n1 + nb)
    P = rng.normal(size=(n0, n1, nb, nb)) + 1j * rng.normal(size=(n0, n1, nb, nb))
    VR = rng.normal(size=(n0, n1, nb, nb)) + 1j * rng.normal(size=(n0, n1, nb, nb))
    got = native.selfenergy_fft_full(VR, P, shift, False)
    ref = oracle.selfenergy_fft_full(VR, P, shift, False)
    assert rel(got, ref) < 1e-12


@pytest.mark.parametrize("n0,n1,nb", [(1, 1, 2), (12, 12, 4), (48, 48, 2), (7, 9, 5), (144, 144, 8)])
def test_exchange_scalar_and_hcp(native, oracle, n0, n1, nb):
    rng = np.random.default_rng(7 + n0 + nb)
    P = rand_herm(rng, (n0, n1, nb, nb))
    VR = _scalar_VR(rng, n0, n1)
    full = native.selfenergy_fft_full(VR, P, False, False)
    hcp = native.selfenergy_fft_full(VR, P, False, True)
    ref = oracle.selfenergy_fft_full(VR, P, False, True)
    assert rel(full, ref) < 1e-12
    assert rel(hcp, ref) < 1e-12


def test_exchange_single_point_definition(native):
    VR = np.array([[[[0.3]]]], dtype=np.complex64)
    P = np.array([[[[1.0 + 0.5j, 0.2], [0.2, 0.8 - 0.1j]]]], dtype=np.complex64)
    np.testing.assert_allclose(native.selfenergy_fft_full(VR, P), -VR * P, rtol=1e-6, atol=1e-6)


def test_exchange_hcp_requires_scalar_kernel(native):
    with pytest.raises(ValueError, match="hermitian_channel_packing"):
        native.selfenergy_fft_full(np.ones((2, 2, 2, 2)), np.ones((2, 2, 2, 2)), False, True)


def test_exchange_layered_full_size_matches_oracle(native, oracle):
    """192^2, nb=8, layer-resolved VR: the benchmark's exchange at full size."""
    args, _P0, _ = workloads.layered(192, n_layers=4, seed=0)
    P = workloads.random_hermitian_density(192, 8, seed=1)
    got = native.selfenergy_fft_full(args["VR"], P, False, False)
    ref = oracle.selfenergy_fft_full(args["VR"], P, False, False)
    assert rel(got, ref) < 1e-12


def test_exchange_complex64_precision(native, oracle):
    import torch

    from cpp_hf_b200 import _lib, _native as nat

    rng = np.random.default_rng(5)
    P = rand_herm(rng, (48, 48, 4, 4))
    VR = rng.normal(size=(48, 48, 4, 4)) + 1j * rng.normal(size=(48, 48, 4, 4))
    P_t = torch.from_numpy(P).cuda()
    VR_t = torch.from_numpy(VR).cuda()
    s32 = nat._exchange(VR_t, P_t, False, False, precision=32).cpu().numpy()
    ref = oracle.selfenergy_fft_full(VR, P, False, False)
    assert rel(s32, ref) < 5e-6
    assert _lib.load() is not None


# ---------------------------------------------------------------------------
# eigh
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("batch,nb", [(1, 1), (5, 2), (64, 3), (300, 8), (17, 13), (9, 16), (4, 24), (3, 64)])
def test_eigh_batched(native, batch, nb):
    rng = np.random.default_rng(batch + nb)
    M = rng.normal(size=(batch, nb, nb)) + 1j * rng.normal(size=(batch, nb, nb))
    w, V = native.eigh_batched(M)
    H = herm(M)
    w_ref = np.linalg.eigvalsh(H)
    scale = np.max(np.abs(w_ref))
    assert np.max(np.abs(w - w_ref)) < 1e-12 * max(scale, 1.0)
    assert np.all(np.diff(w, axis=-1) >= 0)
    rec = (V * w[..., None, :]) @ np.conj(np.swapaxes(V, -1, -2))
    assert np.max(np.abs(rec - H)) < 1e-12 * max(scale, 1.0)
    eye = np.eye(nb)
    assert np.max(np.abs(np.conj(np.swapaxes(V, -1, -2)) @ V - eye)) < 1e-12


def test_eigh_degenerate_and_diagonal(native):
    M = np.zeros((3, 4, 4), dtype=np.complex128)
    M[0] = np.eye(4)
    M[1] = np.diag([3.0, 1.0, 1.0, -2.0])
    M[2] = np.diag([1.0, 1.0, 1.0, 1.0]) + 1e-3 * herm(np.arange(16).reshape(4, 4) * (1 + 1j))
    w, V = native.eigh_batched(M)
    np.testing.assert_allclose(w[0], np.ones(4), atol=1e-15)
    np.testing.assert_allclose(w[1], [-2.0, 1.0, 1.0, 3.0], atol=1e-15)
    rec = (V * w[..., None, :]) @ np.conj(np.swapaxes(V, -1, -2))
    np.testing.assert_allclose(rec, herm(M), atol=1e-13)


@pytest.mark.parametrize("sort", [True, False])
def test_eigh_block_sizes(native, oracle, sort):
    rng = np.random.default_rng(11)
    M = rand_herm(rng, (6, 5, 5))
    M[..., :2, 2:] = 0
    M[..., 2:, :2] = 0
    w, V = native.eigh_block_sizes(M, [2, 3], sort)
    wr, Vr = oracle.eigh_block_sizes(M, [2, 3], sort)
    np.testing.assert_allclose(w, wr, atol=1e-12)
    np.testing.assert_allclose(np.abs(V), np.abs(Vr), atol=1e-10)
    assert native.max_offblock_sizes(M, [2, 3]) == 0.0
    M2 = M.copy()
    M2[..., 0, 4] = 0.25
    assert abs(native.max_offblock_sizes(M2, [2, 3]) - oracle.max_offblock_sizes(M2, [2, 3])) < 1e-15


# ---------------------------------------------------------------------------
# mu
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("nk,nb,T", [(1, 2, 0.1), (16, 6, 0.05), (2304, 2, 0.1), (36864, 8, 0.05)])
def test_find_mu_bisection(native, oracle, nk, nb, T):
    rng = np.random.default_rng(nk + nb)
    bands = rng.normal(size=(nk, nb))
    w = np.full(nk, 1.0 / nk)
    n_e = 0.5 * nb
    mu = native.find_mu_bisection(bands, w, n_e, T, 0)
    mu_ref = oracle.find_mu_bisection(bands, w, n_e, T, 0)
    assert abs(mu - mu_ref) < 1e-12 * max(1.0, abs(mu_ref))


@pytest.mark.parametrize("nk,nb,T,maxiter", [(36864, 8, 0.01, 0), (9216, 4, 0.5, 0), (36864, 8, 0.05, 12),
                                             (36864, 8, 0.05, 45), (40000, 2, 0.002, 0)])
def test_find_mu_bisection_root_replay(native, oracle, nk, nb, T, maxiter):
    """Large multi-block problems, where the GPU runs the first bisection levels
    as multisection rounds, finds the root of N(mu) = n_e by Newton and replays
    the remaining levels against it: the result equals the oracle's sequential
    bisection for short, default and long level counts and cold and hot T."""
    rng = np.random.default_rng(nk + nb + int(1e3 * T) + maxiter)
    bands = rng.normal(size=(nk, nb))
    w = rng.uniform(0.5, 1.5, size=nk)
    w /= w.sum()
    n_e = 0.37 * nb
    mu = native.find_mu_bisection(bands, w, n_e, T, maxiter)
    mu_ref = oracle.find_mu_bisection(bands, w, n_e, T, maxiter)
    assert abs(mu - mu_ref) < 1e-12 * max(1.0, abs(mu_ref))


def test_find_mu_bisection_gapped_spectrum(native, oracle):
    """mu inside a band gap with T well below the gap: N(mu) is flat to rounding
    there, so the GPU keeps exact counts for the levels whose sign is not certain
    (the reference's own decisions are rounding noise there too); the count
    reached must equal n_e and mu must lie in the gap."""
    rng = np.random.default_rng(5)
    nk, nb = 40000, 4
    lower = rng.uniform(-2.0, -1.0, size=(nk, nb // 2))
    upper = rng.uniform(1.0, 2.0, size=(nk, nb // 2))
    bands = np.concatenate([lower, upper], axis=1)
    w = np.full(nk, 1.0 / nk)
    n_e = nb // 2
    T = 0.02
    mu = native.find_mu_bisection(bands, w, n_e, T, 0)
    mu_ref = oracle.find_mu_bisection(bands, w, n_e, T, 0)
    assert -1.0 < mu < 1.0 and -1.0 < mu_ref < 1.0
    occ = 0.5 * (1.0 - np.tanh(0.5 * (bands - mu) / (T + 1e-12)))
    assert abs(float(np.sum(w[:, None] * occ)) - n_e) < 1e-12


def test_find_mu_bisection_cold_limit_hits_target(native, oracle):
    """T -> 0 with the target on a plateau of the count: mu is only defined up to
    the plateau (serial, pairwise and tree sums decide count > n_e differently
    when the count equals n_e to the last bit), so check the count itself, as
    the reference's tests/test_main.py:227-234 does."""
    rng = np.random.default_rng(13)
    bands = rng.normal(size=(10, 3))
    w = np.full(10, 0.1)
    for T in (1e-5, 1e-3):
        mu = native.find_mu_bisection(bands, w, 1.5, T, 0)
        occ = 1.0 / (1.0 + np.exp((bands - mu) / (T + 1e-12)))
        assert abs(float(np.sum(w[:, None] * occ)) - 1.5) < 1e-4


def test_find_mu_bisection_float32_inputs(native, oracle):
    bands = np.array([[[0.0, 1.0]]], dtype=np.float32)
    weights = np.ones((1, 1), dtype=np.float32)
    assert abs(native.find_mu_bisection(bands, weights, 1.0, 0.1) - oracle.find_mu_bisection(
        bands, weights, 1.0, 0.1)) < 1e-12


# ---------------------------------------------------------------------------
# build_fock_apply
# ---------------------------------------------------------------------------

def _hartree_case(nk=3, nb=3, contact=True, seed=4):
    rng = np.random.default_rng(seed)
    w = np.ones((nk, nk)) / (nk * nk)
    h = rand_herm(rng, (nk, nk, nb, nb))
    refP = 0.1 * rand_herm(rng, (nk, nk, nb, nb))
    HH = rng.normal(size=(nb, nb))
    HH = 0.5 * (HH + HH.T)
    Vq = np.full((nk, nk, 1, 1), 0.15)
    ct = None
    if contact:
        Oz = np.diag(np.where(np.arange(nb) % 2 == 0, 1.0, -1.0)).astype(np.complex128)
        Ox = np.roll(np.eye(nb), 1, axis=1).astype(np.complex128)
        ct = [(0.3, Oz, Oz), (-0.1, Ox, Ox.T.copy())]
    args = problem.kernel_args(w, h, Vq, 0.1, include_hartree=True, include_exchange=True,
                               reference_density=refP, hartree_matrix=HH, contact_terms=ct)
    P = rand_herm(rng, (nk, nk, nb, nb))
    return args, P


@pytest.mark.parametrize("contact", [False, True])
@pytest.mark.parametrize("nk,nb", [(3, 3), (12, 4), (9, 8)])
def test_build_fock_apply_hartree_contact_refP(native, oracle, contact, nk, nb):
    args, P = _hartree_case(nk, nb, contact)
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 1e-11
    assert rel(H, Hr) < 1e-12 if np.any(Hr) else np.max(np.abs(H)) == 0
    assert rel(F, Fr) < 1e-11
    assert abs(E - Er) < 1e-11 * max(1.0, abs(Er))


def test_build_fock_layered_no_hcp(native, oracle):
    args, _P0, _ = workloads.layered(24, n_layers=3, seed=3)
    P = workloads.random_hermitian_density(24, 6, seed=2)
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 1e-11 and rel(F, Fr) < 1e-11
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er))


def test_build_fock_project_callback(native):
    args = problem.kernel_args(np.ones((1, 1)), np.eye(2, dtype=np.complex128)[None, None], np.ones((1, 1, 1, 1)), 0.1)
    P = np.zeros((1, 1, 2, 2), dtype=np.complex128)
    _S, _H, F, _E = native.build_fock_apply(args, P, lambda F: np.zeros_like(F))
    np.testing.assert_allclose(F, np.zeros_like(F), atol=0.0)


# ---------------------------------------------------------------------------
# spectral Cayley hooks
# ---------------------------------------------------------------------------

def _skew(rng, shape):
    d = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    return 0.5 * (d - np.conj(np.swapaxes(d, -1, -2)))


@pytest.mark.parametrize("nb", [2, 6, 8, 20])
def test_cayley_hooks_match_lu(native, nb):
    rng = np.random.default_rng(nb)
    d = _skew(rng, (3, 3, nb, nb))
    Ft = rand_herm(rng, (3, 3, nb, nb))
    V, lam = native._cayley_spectral_setup(d)
    Fe = np.conj(np.swapaxes(V, -2, -1)) @ Ft @ V
    eye = np.eye(nb)
    for tau in [0.0, 0.1, 0.5, 1.0, -0.3]:
        A = 0.5 * tau * d
        U_lu = np.linalg.solve(eye + A, eye - A)
        U = native._cayley_unitary_from_spectrum(V, lam, tau)
        np.testing.assert_allclose(U, U_lu, atol=1e-12, rtol=1e-12)
        dg = native._diag_UFU_from_spectrum(V, Fe, lam, tau)
        ref = np.real(np.diagonal(np.conj(np.swapaxes(U_lu, -2, -1)) @ Ft @ U_lu, axis1=-2, axis2=-1))
        np.testing.assert_allclose(dg, ref, atol=1e-12, rtol=1e-12)


# ---------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------

def _dm(mod, args, P0, n_e, max_iter=200, tol_E=1e-10, block_sizes=(), project_fn=None):
    nk1, nk2, nb = P0.shape[0], P0.shape[1], P0.shape[2]
    return mod.solve_dm(args, P0, n_e, max_iter, tol_E, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                        np.empty((0, nk1, nk2, nb, nb), np.complex128), 0.0, 1.0, list(block_sizes),
                        project_fn, True, True, True)


def _scf(mod, args, P0, n_e, max_iter=200, dtol=1e-9, ctol=1e-9, mixing=0.5, level_shift=0.0, project_fn=None):
    return mod.solve_scf(args, P0, n_e, max_iter, dtol, ctol, mixing, level_shift, project_fn, [], "linear",
                         6, 2, 1.0, 0.0, True, True)


def _check_dm(got, ref, e_tol=1e-9, f_tol=1e-8):
    Q, p, D, F, mu, E, n, conv, hE, hG = got
    Qr, pr, Dr, Fr, mur, Er, nr, convr, hEr, hGr = ref
    print(f"iterations gpu {n} oracle {nr}; |dE| {abs(E - Er):.3e}; |dmu| {abs(mu - mur):.3e}")
    assert conv == convr
    assert abs(E - Er) < e_tol * max(1.0, abs(Er))
    # mu is ill-conditioned when it sits in a gap (N(mu) flat); the occupations are not
    assert abs(mu - mur) < 1e-4
    assert rel(p, pr) < f_tol
    assert rel(D, Dr) < f_tol
    assert rel(F, Fr) < f_tol
    assert abs(n - nr) <= max(2, nr // 5)


def test_solve_dm_two_band_tiny(native, oracle):
    w = np.ones((1, 1))
    h = np.zeros((1, 1, 2, 2), dtype=np.complex128)
    h[..., 0, 0], h[..., 1, 1] = -0.5, 0.5
    args = problem.kernel_args(w, h, np.full((1, 1, 1, 1), 0.25), 0.2)
    P0 = np.zeros_like(h)
    _check_dm(_dm(native, args, P0, 1.0, 100, 1e-8), _dm(oracle, args, P0, 1.0, 100, 1e-8))


def test_solve_dm_dirac_12(native, oracle):
    args, P0, n_e = workloads.dirac(12, seed=0)
    _check_dm(_dm(native, args, P0, n_e), _dm(oracle, args, P0, n_e))


def test_solve_dm_layered_small(native, oracle):
    args, P0, n_e = workloads.layered(8, n_layers=2, seed=0)
    _check_dm(_dm(native, args, P0, n_e, tol_E=1e-11), _dm(oracle, args, P0, n_e, tol_E=1e-11))


def test_solve_dm_hartree_contact(native, oracle):
    args, P = _hartree_case(4, 3, True, seed=9)
    n_e = 1.0
    P0 = np.zeros_like(P)
    _check_dm(_dm(native, args, P0, n_e), _dm(oracle, args, P0, n_e))


def test_solve_dm_result_shapes_and_omission(native):
    args, P0, n_e = workloads.dirac(6, seed=0)
    out = native.solve_dm(args, P0, n_e, 50, 1e-8, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                          np.empty((0, 6, 6, 2, 2), np.complex128), 0.0, 1.0, [], None, False, False, False)
    assert out[0] is None and out[2] is None and out[3] is None
    assert out[1].shape == (6, 6, 2)
    assert len(out[8]) == out[6]


def test_solve_dm_rejects_bad_blocks(native):
    args, P0, n_e = workloads.dirac(4, seed=0)
    with pytest.raises(ValueError, match="block_sizes must sum to nb"):
        _dm(native, args, P0, n_e, 5, block_sizes=(1, 2))


def test_solve_dm_project_callback(native, oracle):
    args, P0, n_e = workloads.dirac(6, seed=2)

    def proj(M):  # average with the k -> -k partner (a symmetrising projector)
        return 0.5 * (M + np.roll(np.flip(M, axis=(0, 1)), 1, axis=(0, 1)))

    _check_dm(_dm(native, args, P0, n_e, 100, 1e-9, project_fn=proj),
              _dm(oracle, args, P0, n_e, 100, 1e-9, project_fn=proj), e_tol=1e-8, f_tol=1e-7)


def test_solve_scf_two_band_and_dirac(native, oracle):
    for args, P0, n_e in [workloads.dirac(8, seed=3), workloads.layered(6, n_layers=2, seed=1)]:
        got = _scf(native, args, P0, n_e)
        ref = _scf(oracle, args, P0, n_e)
        print("scf iterations", got[4], ref[4], "dE", abs(got[2] - ref[2]))
        assert got[5] == ref[5]
        assert abs(got[2] - ref[2]) < 1e-9 * max(1.0, abs(ref[2]))
        assert rel(got[0], ref[0]) < 1e-8
        assert rel(got[1], ref[1]) < 1e-8
        assert abs(got[4] - ref[4]) <= 1


def test_solve_scf_level_shift(native, oracle):
    args, P0, n_e = workloads.dirac(6, seed=4)
    got = _scf(native, args, P0, n_e, level_shift=0.2)
    ref = _scf(oracle, args, P0, n_e, level_shift=0.2)
    assert abs(got[2] - ref[2]) < 1e-9 * max(1.0, abs(ref[2]))
    assert abs(got[4] - ref[4]) <= 1


def test_solve_scf_meshgrid_regression_case(native):
    from conftest import GOLDEN

    d = np.load(GOLDEN / "meshgrid_scf_v1.npz")
    args = problem.kernel_args(d["weights"], d["hamiltonian"], d["coulomb_q"], float(d["T"]),
                               include_hartree=True, include_exchange=True,
                               reference_density=d["reference_density"], hartree_matrix=d["hartree_matrix"])
    out = _scf(native, args, np.asarray(d["P0"]), float(d["electrondensity0"]), int(d["max_iter"]),
               float(d["comm_tol"]), float(d["comm_tol"]))
    assert out[5]
    np.testing.assert_allclose(out[0], d["P_expected"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(out[1], d["F_expected"], rtol=1e-6, atol=1e-6)
    assert abs(out[3] - float(d["mu_expected"])) < 1e-6
    assert abs(out[8][0] - float(d["hist_dC_expected"][0])) < 1e-6


def _scf_acc(mod, args, P0, n_e, acc, diis_size=6, diis_start=2, damping=1.0, trust=0.0, max_iter=200, tol=1e-9,
             project_fn=None):
    return mod.solve_scf(args, P0, n_e, max_iter, tol, tol, 0.5, 0.0, project_fn, [], acc, diis_size, diis_start,
                         damping, trust, True, True)


_ACC_CASES = [
    ("dirac8", "diis", 6, 2, 1.0, 0.0, 200), ("dirac8", "diis", 3, 2, 0.7, 0.0, 200),
    ("dirac8", "diis", 4, 3, 1.0, 0.05, 200), ("dirac8", "oda", 6, 2, 1.0, 0.0, 15),
    ("dirac8", "oda", 6, 2, 1.0, 0.02, 15), ("dirac8", "linear", 6, 2, 1.0, 0.03, 30),
    ("layered6", "diis", 3, 2, 0.7, 0.0, 200), ("layered6", "oda", 6, 2, 1.0, 0.0, 15),
    ("layered6", "oda", 6, 2, 1.0, 0.02, 15), ("layered6", "linear", 6, 2, 1.0, 0.03, 30),
]


def _acc_model(case):
    return workloads.dirac(8, seed=3) if case == "dirac8" else workloads.layered(6, n_layers=2, seed=1)


@pytest.mark.parametrize("case,acc,diis_size,diis_start,damping,trust,max_iter", _ACC_CASES)
def test_solve_scf_acceleration_matches_oracle(native, oracle, case, acc, diis_size, diis_start, damping, trust,
                                                max_iter):
    """C-DIIS (history ring, B matrix from the new residual's inner products,
    complete-pivoting solve with the rank test, extrapolated Fock), ODA (extra
    build at P_new, analytic step) and the trust-radius clip against the oracle's
    restatement of solver_scf.hpp:253-428: same iteration counts and energies.  ODA
    and the clipped linear runs stall on these models (the reference's ODA takes
    lambda = 0 once c1, c2 reach the rounding level), so they are compared over
    their first iterations."""
    args, P0, n_e = _acc_model(case)
    got = _scf_acc(native, args, P0, n_e, acc, diis_size, diis_start, damping, trust, max_iter=max_iter)
    ref = _scf_acc(oracle, args, P0, n_e, acc, diis_size, diis_start, damping, trust, max_iter=max_iter)
    print(f"scf {case} {acc} size {diis_size} start {diis_start} damp {damping} trust {trust}: iterations gpu "
          f"{got[4]} oracle {ref[4]}, |dE| {abs(got[2] - ref[2]):.2e}")
    assert got[5] == ref[5]
    assert abs(got[2] - ref[2]) < 1e-9 * max(1.0, abs(ref[2]))
    assert rel(got[0], ref[0]) < 1e-7
    assert abs(got[4] - ref[4]) <= 1
    # the energy history agrees closely but not to the last digits: a DIIS
    # extrapolation amplifies rounding-level differences for a few iterations
    n = min(len(got[6]), len(ref[6]))
    np.testing.assert_allclose(got[6][:n], ref[6][:n], rtol=1e-6, atol=1e-10)


def test_solve_scf_diis_sensitive_model_reaches_oracle_energy(native, oracle):
    """Undamped C-DIIS on the two-layer model is sensitive to rounding (GPU and
    oracle sum in different orders, and the extrapolation amplifies the
    difference): both converge to the same energy in different iteration counts."""
    args, P0, n_e = _acc_model("layered6")
    got = _scf_acc(native, args, P0, n_e, "diis", 6, 2, 1.0, 0.0, max_iter=400)
    ref = _scf_acc(oracle, args, P0, n_e, "diis", 6, 2, 1.0, 0.0, max_iter=400)
    print(f"layered6 DIIS: iterations gpu {got[4]} oracle {ref[4]}, |dE| {abs(got[2] - ref[2]):.2e}")
    assert got[5] and ref[5]
    assert abs(got[2] - ref[2]) < 1e-9 * max(1.0, abs(ref[2]))
    assert rel(got[0], ref[0]) < 1e-6


def test_solve_scf_diis_meshgrid_regression_case(native, oracle):
    """The reference's stored SCF case (Hartree, exchange, reference density) with
    C-DIIS: GPU against the oracle."""
    from conftest import GOLDEN

    d = np.load(GOLDEN / "meshgrid_scf_v1.npz")
    args = problem.kernel_args(d["weights"], d["hamiltonian"], d["coulomb_q"], float(d["T"]),
                               include_hartree=True, include_exchange=True,
                               reference_density=d["reference_density"], hartree_matrix=d["hartree_matrix"])
    P0, n_e = np.asarray(d["P0"]), float(d["electrondensity0"])
    got = _scf_acc(native, args, P0, n_e, "diis", max_iter=60, tol=1e-8)
    ref = _scf_acc(oracle, args, P0, n_e, "diis", max_iter=60, tol=1e-8)
    print(f"meshgrid DIIS: iterations gpu {got[4]} oracle {ref[4]}, |dE| {abs(got[2] - ref[2]):.2e}")
    assert got[5] and ref[5]
    assert abs(got[2] - ref[2]) < 1e-9 * max(1.0, abs(ref[2]))
    assert abs(got[4] - ref[4]) <= 1


def test_solve_scf_rejects_bad_diis_size(native):
    args, P0, n_e = workloads.dirac(4, seed=0)
    with pytest.raises(ValueError, match="diis_size"):
        _scf_acc(native, args, P0, n_e, "diis", diis_size=0)


def test_solve_scf_rejects_unknown_acceleration(native):
    args, P0, n_e = workloads.dirac(4, seed=0)
    with pytest.raises(ValueError, match="acceleration"):
        native.solve_scf(args, P0, n_e, 5, 1e-6, 1e-6, 0.5, 0.0, None, [], "bogus", 6, 2, 1.0, 0.0, True, True)


# ---------------------------------------------------------------------------
# switched precision (complex64 exchange, then complex128)
# ---------------------------------------------------------------------------

def _mixed(args, switch=1e-5):
    a = dict(args)
    a["exchange_precision"] = "mixed"
    a["mixed_switch"] = switch
    return a


@pytest.mark.parametrize("case", ["dirac16", "layered12"])
def test_solve_dm_mixed_precision_reaches_fp64_energy(native, oracle, case):
    args, P0, n_e = workloads.dirac(16, seed=5) if case == "dirac16" else workloads.layered(12, n_layers=4, seed=2)
    ref = _dm(oracle, args, P0, n_e, 300, 1e-11)
    got = _dm(native, _mixed(args), P0, n_e, 300, 1e-11)
    plain = _dm(native, args, P0, n_e, 300, 1e-11)
    print(f"{case}: iterations mixed {got[6]} fp64 {plain[6]} oracle {ref[6]}; "
          f"|dE| mixed {abs(got[5] - ref[5]):.3e} fp64 {abs(plain[5] - ref[5]):.3e}")
    assert got[7] and ref[7]
    # converged energies within 1e-9 of the FP64 oracle (the switched form's bar)
    assert abs(got[5] - ref[5]) < 1e-9 * max(1.0, abs(ref[5]))
    assert rel(got[2], ref[2]) < 1e-4
    # the gradient history is recorded for both phases; the first iterations ran
    # the complex64 exchange, so their energies differ from the FP64 run's
    assert len(got[9]) == got[6]
    assert got[8][0] != plain[8][0]
    assert abs(got[8][0] - plain[8][0]) < 1e-5 * max(1.0, abs(plain[8][0]))


def test_solve_dm_mixed_rejects_complex64_kernel(native):
    args, P0, n_e = workloads.dirac(4, seed=0)
    a = _mixed(args)
    a["exchange_precision"] = "bogus"
    with pytest.raises(ValueError, match="exchange_precision"):
        _dm(native, a, P0, n_e, 5)


def test_solve_scf_mixed_precision_reaches_fp64_energy(native, oracle):
    args, P0, n_e = workloads.dirac(12, seed=3)
    ref = _scf(oracle, args, P0, n_e, 300, 1e-10, 1e-10)
    got = _scf(native, _mixed(args), P0, n_e, 300, 1e-10, 1e-10)
    print(f"scf iterations mixed {got[4]} oracle {ref[4]}; |dE| {abs(got[2] - ref[2]):.3e}")
    assert got[5] and ref[5]
    # the second iteration (the first with a non-zero density) ran the complex64 exchange
    assert got[6][1] != ref[6][1]
    assert abs(got[6][1] - ref[6][1]) < 1e-5 * max(1.0, abs(ref[6][1]))
    assert abs(got[2] - ref[2]) < 1e-9 * max(1.0, abs(ref[2]))
    assert rel(got[0], ref[0]) < 1e-7


@pytest.mark.parametrize("layers", [5, 7, 9])
def test_solve_dm_generic_team_path_matches_oracle(native, oracle, layers):
    """nb = 10, 14 (warp teams) and 18 (CTA team): the general per-k kernels follow the
    oracle's trajectory (energy history of 30 iterations)."""
    args, P0, n_e = workloads.layered(6, n_layers=layers, seed=4)
    got = native.solve_dm(args, P0, n_e, 30, 0.0, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                          np.empty((0, 6, 6, 2 * layers, 2 * layers), np.complex128), 0.0, 1.0, [], None,
                          False, True, False)
    ref = oracle.solve_dm(args, P0, n_e, 30, 0.0, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                          np.empty((0, 6, 6, 2 * layers, 2 * layers), np.complex128), 0.0, 1.0, [], None,
                          False, True, False)
    d = np.abs(np.asarray(got[8]) - np.asarray(ref[8]))
    print(f"nb={2 * layers}: energy history |dE| per iteration {np.array2string(d[:8], precision=2)} ... max {d.max():.2e}")
    assert d.max() < 1e-9 * max(1.0, float(np.max(np.abs(ref[8]))))


# ---------------------------------------------------------------------------
# resample_kgrid_2d (utils.hpp:120-176)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n_old,n_new,inner", [(12, 18, (4, 4)), (18, 12, (4, 4)), (7, 13, ()), (16, 16, (2, 2)),
                                               (1, 3, (3,)), (24, 48, (8, 8)), (48, 24, (2, 2)), (5, 4, (6, 6))])
def test_resample_kgrid_2d_matches_oracle(native, oracle, n_old, n_new, inner):
    """Periodic linear resampling of the two leading k axes: the GPU evaluates both
    passes per element in the reference's order without fused multiply-adds, so it
    equals the oracle's two-pass result bit for bit."""
    rng = np.random.default_rng(n_old * 100 + n_new)
    x = rng.normal(size=(n_old, n_old) + inner) + 1j * rng.normal(size=(n_old, n_old) + inner)
    got = native.resample_kgrid_2d(x, n_new)
    ref = oracle.resample_kgrid_2d(x, n_new)
    assert got.shape == ref.shape == (n_new, n_new) + inner
    np.testing.assert_array_equal(got, ref)


def test_resample_kgrid_2d_errors(native):
    with pytest.raises(ValueError, match="need >= 2 dims"):
        native.resample_kgrid_2d(np.zeros(4, np.complex128), 8)
    with pytest.raises(ValueError, match="square"):
        native.resample_kgrid_2d(np.zeros((4, 5), np.complex128), 8)

