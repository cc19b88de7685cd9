"""GPU: the solvers' CUDA-graph path against their launch-by-launch path.

With ``solve_graphs`` (the default) solve() replays one captured graph per
iteration and solve_scf() with linear mixing does too; for nb <= 8 the SCF
graph path also writes the linear mix (solver_scf.hpp:395-401) from the
residual pass instead of a separate mix kernel, with the same per-element
arithmetic.  Both paths must give the same trajectory: same iteration counts
and the same energies, densities and chemical potentials to rounding.
"""

from __future__ import annotations

import numpy as np
import pytest

from cpp_hf_b200 import workloads

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def _scf(mod, args, P0, n_e):
    return mod.solve_scf(args, P0, n_e, 200, 1e-9, 1e-9, 0.5, 0.0, None, [], "linear", 6, 2, 1.0, 0.0, True, True)


def _dm(mod, args, P0, n_e):
    empty = np.empty((0,) + P0.shape, np.complex128)
    return mod.solve_dm(args, P0, n_e, 200, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0, 1.0,
                        [], None, True, True, True)


@pytest.mark.parametrize("n,layers", [(16, 4), (24, 2)])
def test_scf_graph_path_matches_launch_path(native, n, layers):
    args, P0, n_e = workloads.layered(n, n_layers=layers, seed=n)
    D_g, F_g, E_g, mu_g, it_g, conv_g, hE_g, hD_g, hC_g = _scf(native, dict(args, solve_graphs=True), P0, n_e)
    D_e, F_e, E_e, mu_e, it_e, conv_e, hE_e, hD_e, hC_e = _scf(native, dict(args, solve_graphs=False), P0, n_e)
    assert it_g == it_e and conv_g == conv_e
    assert it_g > 2
    assert abs(E_g - E_e) <= 1e-13 * max(1.0, abs(E_e))
    assert rel(hE_g, hE_e) <= 1e-13
    assert rel(hD_g, hD_e) <= 1e-9
    assert rel(D_g, D_e) <= 1e-12
    assert rel(F_g, F_e) <= 1e-12
    assert abs(mu_g - mu_e) <= 1e-12 * max(1.0, abs(mu_e))


@pytest.mark.parametrize("n", [16])
def test_dm_graph_path_matches_launch_path(native, n):
    args, P0, n_e = workloads.layered(n, n_layers=4, seed=n + 1)
    out_g = _dm(native, dict(args, solve_graphs=True), P0, n_e)
    out_e = _dm(native, dict(args, solve_graphs=False), P0, n_e)
    Q_g, p_g, D_g, F_g, mu_g, E_g, it_g, conv_g, hE_g, hG_g = out_g
    Q_e, p_e, D_e, F_e, mu_e, E_e, it_e, conv_e, hE_e, hG_e = out_e
    assert it_g == it_e and conv_g == conv_e
    assert abs(E_g - E_e) <= 1e-13 * max(1.0, abs(E_e))
    assert rel(hE_g, hE_e) <= 1e-13
    assert rel(D_g, D_e) <= 1e-12
    assert rel(p_g, p_e) <= 1e-12
