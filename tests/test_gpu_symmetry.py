"""GPU parity of the device symmetry projector (cpp_hf src/cpp_hf/symmetry.py) and of
symmetric solves that apply it on the device."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN
from cpp_hf_b200 import symmetry, workloads

pytestmark = pytest.mark.gpu


def _cases(G, S, U):
    from test_oracle_pins import _symmetry_kwargs

    return _symmetry_kwargs(G, S, U)


def test_device_projector_matches_reference_vectors():
    """Every configuration of the golden fixture made by the reference's
    make_project_fn: unitary, spatial ('mod' and 'flip' with one axis), both,
    time reversal ('mod' and 'flip'), and all together."""
    d = np.load(GOLDEN / "symmetry_ref.npz")
    for name, kw in _cases(d["in.G"], d["in.S"], d["in.U"]).items():
        got = symmetry.make_project_fn(**kw)(d["in.A"])
        np.testing.assert_allclose(got, d[f"{name}.out"], rtol=0, atol=1e-13, err_msg=name)


def _reference_style_projector(G=None, S=None, U=None, s_k_conv="mod", s_k_axes=(0, 1), t_k_conv="mod",
                               t_k_axes=(0, 1)):
    """A closure shaped like the one cpp_hf.symmetry.make_project_fn returns (same
    free variables, module and qualified name), numpy-valued."""
    from oracle import symmetry_np

    ref = symmetry_np.make_project_fn(unitary_group=G, spatial_group=S, spatial_k_convention=s_k_conv,
                                      spatial_k_flip_axes=s_k_axes, time_reversal_U=U,
                                      time_reversal_k_convention=t_k_conv, time_reversal_k_flip_axes=t_k_axes)

    def project(A):
        _ = (G, S, U, s_k_conv, s_k_axes, t_k_conv, t_k_axes)
        return ref(A)

    project.__module__ = "cpp_hf.symmetry"
    project.__qualname__ = "make_project_fn.<locals>.project"
    return project


def test_reference_projector_is_recognised():
    d = np.load(GOLDEN / "symmetry_ref.npz")
    fn = _reference_style_projector(G=d["in.G"], S=d["in.S"], U=d["in.U"], s_k_axes=(1,))
    dp = symmetry.device_projector(fn)
    assert isinstance(dp, symmetry.DeviceProjector)
    np.testing.assert_allclose(dp(d["in.A"]), d["all.out"], rtol=0, atol=1e-13)
    assert symmetry.device_projector(lambda A: A) is None


def _dirac_symmetry(n):
    """Two-band Dirac model with its inversion symmetry sigma_z H(-k) sigma_z = H(k)
    (a spatial group with the 'mod' k convention), exact up to the seeded noise,
    which the projector averages away."""
    args, P0, n_e = workloads.dirac(n, seed=6)
    sz = np.diag([1.0, -1.0]).astype(np.complex128)
    return args, P0, n_e, dict(spatial_group=sz[None])


@pytest.mark.parametrize("solver", ["dm", "scf"])
def test_symmetric_solve_with_device_projector_matches_oracle(native, oracle, solver):
    """A solve whose project_fn is the device projector (applied inside the solve
    on the device) against the oracle solve with the NumPy projector."""
    from oracle import symmetry_np

    args, P0, n_e, kw = _dirac_symmetry(8)
    dev = symmetry.make_project_fn(**kw)
    host = symmetry_np.make_project_fn(**kw)
    if solver == "dm":
        def run(mod, proj):
            return mod.solve_dm(args, P0, n_e, 200, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                                np.empty((0, 8, 8, 2, 2), np.complex128), 0.0, 1.0, [], proj, True, True, True)
        got, ref = run(native, dev), run(oracle, host)
        E, Er, n, nr, D, Dr = got[5], ref[5], got[6], ref[6], got[2], ref[2]
    else:
        def run(mod, proj):
            return mod.solve_scf(args, P0, n_e, 200, 1e-9, 1e-9, 0.5, 0.0, proj, [], "linear", 6, 2, 1.0, 0.0,
                                 True, True)
        got, ref = run(native, dev), run(oracle, host)
        E, Er, n, nr, D, Dr = got[2], ref[2], got[4], ref[4], got[0], ref[0]
    print(f"symmetric {solver}: iterations gpu {n} oracle {nr}, |dE| {abs(E - Er):.2e}")
    assert abs(E - Er) < 1e-9 * max(1.0, abs(Er))
    assert np.max(np.abs(D - Dr)) < 1e-7
    assert abs(n - nr) <= max(2, nr // 5)
