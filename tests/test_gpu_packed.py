"""GPU: the Hermitian-packed Fock build (nb(nb+1)/2 channels, assembly fused into
the last FFT pass) against the oracle's full-channel build, and against the
GPU's own full-channel path.

The packed path runs when V(q) is Hermitian at every q and the density is
Hermitian (cpp_hf's exchange_hcp packing, selfenergy.hpp:119-171, extended to
orbital-resolved V): for build_fock_apply when kernel_args carries
``hermitian_density=True`` (or exchange_hcp with a scalar VR), for every solve
whose kernel qualifies.  Tolerances: 1e-11 relative for Sigma and F (the
full path's bar), 1e-10 relative for the energy, 5e-6 for complex64 passes.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rand_herm
from cpp_hf_b200 import problem, workloads

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _orbital_case(n0, n1, nb, seed, refP=False, hartree=False, contact=False, complex_v=False):
    """Real symmetric (or, with complex_v, Hermitian) orbital-resolved V(q) on an n0 x n1 mesh."""
    rng = np.random.default_rng(seed)
    k0 = -np.pi + 2 * np.pi * np.arange(n0) / n0
    k1 = -np.pi + 2 * np.pi * np.arange(n1) / n1
    kx, ky = np.meshgrid(k0, k1, indexing="ij")
    q = np.sqrt(kx ** 2 + ky ** 2)
    idx = np.arange(nb)
    dist = np.abs(idx[:, None] - idx[None, :])
    Vq = (2 * np.pi / (q + 0.05))[..., None, None] * np.exp(-0.3 * q[..., None, None] * dist)
    if complex_v:
        Vq = Vq * np.exp(1j * 0.2 * (idx[:, None] - idx[None, :]))  # Hermitian at every q
    w = np.full((n0, n1), 1.0 / (n0 * n1))
    h = rand_herm(rng, (n0, n1, nb, nb))
    kw = {}
    if refP:
        kw["reference_density"] = 0.1 * rand_herm(rng, (n0, n1, nb, nb))
    if hartree:
        HH = rng.normal(size=(nb, nb))
        kw["hartree_matrix"] = 0.5 * (HH + HH.T)
    if contact:
        Oz = np.diag(np.where(idx % 2 == 0, 1.0, -1.0)).astype(np.complex128)
        Ox = np.roll(np.eye(nb), 1, axis=1).astype(np.complex128)
        kw["contact_terms"] = [(0.3, Oz, Oz), (-0.1, Ox, Ox.T.copy())]
    args = problem.kernel_args(w, h, Vq, 0.07, include_hartree=hartree, include_exchange=True, **kw)
    P = rand_herm(rng, (n0, n1, nb, nb))
    return args, P


@pytest.mark.parametrize("n0,n1,nb", [(12, 12, 2), (16, 12, 3), (24, 24, 4), (12, 18, 5), (36, 36, 6),
                                      (9, 24, 7), (48, 48, 8), (1, 8, 8), (6, 1, 3)])
def test_packed_build_matches_oracle(native, oracle, n0, n1, nb):
    args, P = _orbital_case(n0, n1, nb, seed=n0 * 100 + nb)
    args["hermitian_density"] = True
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 1e-11
    assert rel(F, Fr) < 1e-11
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er))


@pytest.mark.parametrize("nb", [3, 8])
def test_packed_build_refP_hartree_contact(native, oracle, nb):
    args, P = _orbital_case(12, 12, nb, seed=7 + nb, refP=True, hartree=True, contact=True)
    args["hermitian_density"] = True
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 1e-11
    assert rel(H, Hr) < 1e-12
    assert rel(F, Fr) < 1e-11
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er))


def test_packed_build_complex_hermitian_v(native, oracle):
    """V(q) Hermitian but not real: VR_ba(R) = conj VR_ab(-R) still holds."""
    args, P = _orbital_case(24, 24, 4, seed=5, complex_v=True)
    args["hermitian_density"] = True
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 1e-11 and rel(F, Fr) < 1e-11
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er))


def test_non_hermitian_v_keeps_full_path(native, oracle):
    """A VR that breaks the symmetry is detected and built with all nb*nb channels."""
    from cpp_hf_b200._native import _DeviceKernel

    args, P = _orbital_case(12, 12, 3, seed=9)
    rng = np.random.default_rng(1)
    shape = args["VR"].shape
    args["VR"] = args["VR"] + 0.05 * (rng.normal(size=shape) + 1j * rng.normal(size=shape))
    args["hermitian_density"] = True
    assert not _DeviceKernel(args).v_hermitian()
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 1e-11 and rel(F, Fr) < 1e-11


def test_packed_equals_full_path_layered_192():
    """Full size (192 x 192, nb = 8): the packed build equals the full-channel build."""
    import torch

    from cpp_hf_b200.fock_builder import FockBuilder

    args, _P0, _ = workloads.layered(192, n_layers=4, seed=0)
    P = torch.from_numpy(workloads.random_hermitian_density(192, 8, seed=1)).cuda()
    P = 0.5 * (P + P.conj().transpose(-1, -2))
    full = FockBuilder(args, precision=64)
    packed = FockBuilder(args, precision=64, hermitian_density=True)
    assert packed.packed and not full.packed
    _S0, F0, E0 = [x.clone() for x in full.build(P)]
    _S1, F1, E1 = packed.build(P)
    torch.cuda.synchronize()
    assert float((F1 - F0).abs().max() / F0.abs().max()) < 1e-12
    assert abs(float(E1) - float(E0)) < 1e-11 * abs(float(E0))


def test_packed_complex64_build(native, oracle):
    args, P = _orbital_case(48, 48, 8, seed=3)
    args["hermitian_density"] = True
    args["exchange_precision"] = 32
    S, H, F, E = native.build_fock_apply(args, P, None)
    Sr, Hr, Fr, Er = oracle.build_fock_apply(args, P, None)
    assert rel(S, Sr) < 5e-6
    assert rel(F, Fr) < 5e-6
    assert abs(E - Er) < 5e-6 * max(1.0, abs(Er))


@pytest.mark.parametrize("kind", ["dm", "scf"])
def test_packed_solves_match_full_path(native, kind):
    """Solves take the packed build when V allows it; the full path gives the same answer."""
    args, P0, n_e = workloads.layered(24, n_layers=4, seed=2)
    empty = np.empty((0, 24, 24, 8, 8), np.complex128)
    res = {}
    for packing in (True, False):
        a = dict(args, hermitian_packing=packing)
        if kind == "dm":
            r = native.solve_dm(a, P0, n_e, 300, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0,
                                1.0, [], None, False, True, True)
            res[packing] = (r[5], r[6], r[2])
        else:
            r = native.solve_scf(a, P0, n_e, 300, 1e-9, 1e-9, 0.5, 0.0, None, [], "linear", 6, 2, 1.0, 0.0, True,
                                 True)
            res[packing] = (r[2], r[4], r[0])
    (e1, n1, d1), (e0, n0, d0) = res[True], res[False]
    assert n1 == n0
    assert abs(e1 - e0) < 1e-10 * abs(e0)
    assert rel(d1, d0) < 1e-8
