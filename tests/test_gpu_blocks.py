"""GPU: the block-diagonal fast path of the solvers (block_sizes) against the oracle.

The reference diagonalises block by block when the problem keeps the orbital
blocks: solve() checks h, refP and the contact operators once and F after the
first build (solver_dm.hpp:80-115, 403-450, 622-624); solve_scf() checks each
Fock matrix (solver_scf.hpp:96-124).  Eigenvalues then come block by block
(not globally sorted), which is visible in the occupations solve() returns.
The case below is the layered model with the interlayer hopping switched off
and Hermitian noise inside each layer's 2 x 2 block only, so the layers stay
decoupled and block_sizes = [2, 2, 2, 2] holds throughout.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rand_herm
from cpp_hf_b200 import problem, workloads

pytestmark = pytest.mark.gpu

BLOCKS = [2, 2, 2, 2]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _decoupled_layers(n, seed, couple=0.0):
    h, Vq, w = workloads.layered_model(n, n_layers=4, seed=seed, gamma1=0.0, noise=0.0)
    rng = np.random.default_rng(seed)
    for l in range(4):
        s = slice(2 * l, 2 * l + 2)
        h[..., s, s] += rand_herm(rng, (n, n, 2, 2), scale=0.005)
    if couple:
        h[..., 0, 2] += couple
        h[..., 2, 0] += couple
    args = problem.kernel_args(w, h, Vq, 0.05, include_exchange=True, include_hartree=False)
    return args, np.zeros_like(h), 4.0 * float(np.sum(w))


def _dm(mod, args, P0, n_e, blocks):
    empty = np.empty((0,) + P0.shape, np.complex128)
    return mod.solve_dm(args, P0, n_e, 300, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0, 1.0,
                        blocks, None, True, True, True)


def _scf(mod, args, P0, n_e, blocks):
    return mod.solve_scf(args, P0, n_e, 300, 1e-9, 1e-9, 0.5, 0.0, None, blocks, "linear", 6, 2, 1.0, 0.0, True,
                         True)


@pytest.mark.parametrize("n", [12, 16])
def test_solve_dm_block_path_matches_oracle(native, oracle, n):
    args, P0, n_e = _decoupled_layers(n, seed=n)
    Q, p, D, F, mu, E, it, conv, hE, hG = _dm(native, args, P0, n_e, BLOCKS)
    Qr, pr, Dr, Fr, mur, Er, itr, convr, hEr, hGr = _dm(oracle, args, P0, n_e, BLOCKS)
    assert it == itr and conv == convr
    assert abs(E - Er) < 1e-9 * abs(Er)
    # eigenvalues (and so occupations) block by block, as the reference orders them
    assert float(np.max(np.abs(p - pr))) < 1e-8
    assert rel(D, Dr) < 1e-8 and rel(F, Fr) < 1e-8
    # Q stays block-diagonal
    mask = np.ones((8, 8), bool)
    for l in range(4):
        mask[2 * l:2 * l + 2, 2 * l:2 * l + 2] = False
    assert float(np.max(np.abs(Q[..., mask]))) < 1e-12


def test_solve_dm_block_sizes_ignored_when_h_couples_blocks(native, oracle):
    args, P0, n_e = _decoupled_layers(12, seed=3, couple=0.05)
    r = _dm(native, args, P0, n_e, BLOCKS)
    rr = _dm(oracle, args, P0, n_e, BLOCKS)
    assert r[6] == rr[6]
    assert abs(r[5] - rr[5]) < 1e-9 * abs(rr[5])
    assert float(np.max(np.abs(np.sort(r[1], axis=-1) - np.sort(rr[1], axis=-1)))) < 1e-8


@pytest.mark.parametrize("blocks", [BLOCKS, [4, 4]])
def test_solve_scf_block_path_matches_oracle(native, oracle, blocks):
    args, P0, n_e = _decoupled_layers(12, seed=5)
    D, F, E, mu, it, conv, hE, hD, hC = _scf(native, args, P0, n_e, blocks)
    Dr, Fr, Er, mur, itr, convr, hEr, hDr, hCr = _scf(oracle, args, P0, n_e, blocks)
    assert it == itr and conv == convr
    assert abs(E - Er) < 1e-9 * abs(Er)
    assert rel(D, Dr) < 1e-8 and rel(F, Fr) < 1e-8
