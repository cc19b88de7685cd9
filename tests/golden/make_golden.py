"""Generate the committed golden fixtures in ``tests/golden/`` from the reference.

Run where a checkout of the reference is present, its root directory given
by the ``CPPHF_REFERENCE`` environment variable (required, no default):

    CPPHF_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Writes

* ``meshgrid_scf_v1.npz``: inputs and stored results of the reference's SCF
  regression case ``tests/data/meshgrid_regression_case_v1.npz`` (12x12 mesh,
  nb=4, Hartree + exchange + reference density, linear mixing 0.5).  The
  stored energies use the v1 convention ``Re Tr[h P + (Sigma + H) P / 2]``.
* ``kernel_args_ref.npz``: ``kernel_args`` dicts produced by the reference's
  own ``HartreeFockKernel`` + ``_kernel_args_for_native`` for small seeded
  problems (scalar / layer-resolved interaction, Hartree, contact terms), used
  to pin ``cpp_hf_b200.problem.kernel_args`` (the VR phase convention).
* ``superlattice_ref.npz``: the extended-grid layout and superlattice_*
  kernel_args of a small plane-wave problem from the reference's
  ``build_extended_layout`` + ``SuperlatticeHartreeFockKernel``, used to pin
  ``cpp_hf_b200.superlattice``.

The reference's Python layer needs a ``_native`` module only for the
embedded-reference option, which these cases do not use; the oracle is
installed as a stand-in so the package imports.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
def _reference_root() -> Path:
    root = os.environ.get("CPPHF_REFERENCE")
    if not root:
        raise SystemExit("set CPPHF_REFERENCE to the root of a cpp_hf checkout")
    return Path(root)


REF = _reference_root()


def _ref_cases():
    """Small seeded problems built through the reference's HartreeFockKernel."""
    import cpp_hf
    from cpp_hf.solver import _kernel_args_for_native
    from cpp_hf_b200 import workloads

    out = {}
    # Dirac 12x12 with scalar real V -> HCP flag on.
    rng = np.random.default_rng(11)
    n = 12
    k = workloads.kgrid(n)
    kx, ky = np.meshgrid(k, k, indexing="ij")
    q = np.sqrt(kx ** 2 + ky ** 2)
    h2 = rng.normal(size=(n, n, 2, 2)) + 1j * rng.normal(size=(n, n, 2, 2))
    h2 = 0.5 * (h2 + np.conj(np.swapaxes(h2, -1, -2)))
    V1 = (2 * np.pi / (q + 0.05) * np.tanh(5 * q))[..., None, None]
    w = np.full((n, n), 1.0 / n ** 2)
    out["scalar"] = dict(weights=w, hamiltonian=h2, coulomb_q=V1, T=0.1)
    # Layer-resolved V, nb=4, odd mesh, Hartree + refP + contact term.
    n = 9
    k = workloads.kgrid(n)
    kx, ky = np.meshgrid(k, k, indexing="ij")
    q = np.sqrt(kx ** 2 + ky ** 2)
    h4 = rng.normal(size=(n, n, 4, 4)) + 1j * rng.normal(size=(n, n, 4, 4))
    h4 = 0.5 * (h4 + np.conj(np.swapaxes(h4, -1, -2)))
    lay = np.arange(4) // 2
    V4 = (2 * np.pi / (q + 0.05))[..., None, None] * np.exp(
        -0.3 * q[..., None, None] * np.abs(lay[:, None] - lay[None, :]))
    refP = rng.normal(size=(n, n, 4, 4)) + 1j * rng.normal(size=(n, n, 4, 4))
    refP = 0.1 * (refP + np.conj(np.swapaxes(refP, -1, -2)))
    HH = rng.normal(size=(4, 4))
    HH = 0.5 * (HH + HH.T)
    Oz = np.diag([1.0, -1.0, 1.0, -1.0]).astype(np.complex128)
    w9 = rng.uniform(0.5, 1.5, size=(n, n))
    out["layered"] = dict(weights=w9, hamiltonian=h4, coulomb_q=V4, T=0.05,
                          include_hartree=True, reference_density=refP, hartree_matrix=HH,
                          contact_terms=[(0.3, Oz, Oz)])
    arrays = {}
    for name, kw in out.items():
        kern = cpp_hf.HartreeFockKernel(**kw)
        args = _kernel_args_for_native(kern)
        for key, val in kw.items():
            if key == "contact_terms":
                arrays[f"{name}.in.contact_g"] = np.array([t[0] for t in val])
                arrays[f"{name}.in.contact_Oi"] = np.stack([t[1] for t in val])
                arrays[f"{name}.in.contact_Oj"] = np.stack([t[2] for t in val])
            else:
                arrays[f"{name}.in.{key}"] = np.asarray(val)
        for key, val in args.items():
            arrays[f"{name}.out.{key}"] = np.asarray(val)
    return arrays


def _superlattice_case():
    """Layout + kernel_args of a small superlattice problem built through the
    reference's build_extended_layout and SuperlatticeHartreeFockKernel."""
    from cpp_hf.solver import _kernel_args_for_native
    from cpp_hf.superlattice import SuperlatticeHartreeFockKernel, build_extended_layout
    from cpp_hf_b200 import superlattice as sl

    g, B = sl._triangular_shells(7)
    n = 6
    V = lambda q: 2 * np.pi * 0.5 / (q + 0.05) * np.tanh(5 * q)  # noqa: E731
    layout = build_extended_layout(g, B, n, n, V, 1.0 / n ** 2)
    rng = np.random.default_rng(5)
    D = 2 * g.shape[0]
    h = rng.normal(size=(n, n, D, D)) + 1j * rng.normal(size=(n, n, D, D))
    h = 0.5 * (h + np.conj(np.swapaxes(h, -1, -2)))
    HH_GG = rng.uniform(0.0, 1.0, size=(g.shape[0],) * 2)
    HH_GG = 0.5 * (HH_GG + HH_GG.T)
    np.fill_diagonal(HH_GG, 0.0)
    kern = SuperlatticeHartreeFockKernel(np.full((n, n), 1.0 / n ** 2), h, layout, HH_GG=HH_GG, T=0.05,
                                         hartree_degeneracy=2.0)
    args = _kernel_args_for_native(kern)
    arrays = {"in.g_frac": g, "in.B": B, "in.n": np.array(n), "in.h": h, "in.HH_GG": HH_GG,
              "in.w_scalar": np.array(1.0 / n ** 2)}
    for key, val in args.items():
        arrays[f"out.{key}"] = np.asarray(val)
    return arrays


def _symmetry_cases():
    """Inputs and outputs of the reference's make_project_fn (src/cpp_hf/symmetry.py)
    for the group / spatial / time-reversal combinations and both k conventions."""
    from cpp_hf.symmetry import make_project_fn

    rng = np.random.default_rng(11)
    n1, n2, nb = 6, 5, 4
    A = rng.normal(size=(n1, n2, nb, nb)) + 1j * rng.normal(size=(n1, n2, nb, nb))

    def unitary(m):
        q, _ = np.linalg.qr(rng.normal(size=(m, m)) + 1j * rng.normal(size=(m, m)))
        return q

    G = np.stack([np.eye(nb), unitary(nb), unitary(nb)])
    S = np.stack([unitary(nb), unitary(nb)])
    U = unitary(nb)
    cases = {
        "unitary": dict(unitary_group=G),
        "spatial_mod": dict(spatial_group=S),
        "spatial_flip_axis0": dict(spatial_group=S, spatial_k_convention="flip", spatial_k_flip_axes=(0,)),
        "combined": dict(unitary_group=G, spatial_group=S),
        "tr_mod": dict(time_reversal_U=U),
        "tr_flip_axis1": dict(time_reversal_U=U, time_reversal_k_convention="flip", time_reversal_k_flip_axes=(1,)),
        "all": dict(unitary_group=G, spatial_group=S, time_reversal_U=U, spatial_k_flip_axes=(1,)),
    }
    arrays = {"in.A": A, "in.G": G, "in.S": S, "in.U": U}
    for name, kw in cases.items():
        arrays[f"{name}.out"] = make_project_fn(**kw)(A)
    return arrays


def main():
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REF / "src"))
    from oracle import native_np

    sys.modules["cpp_hf._native"] = native_np

    d = np.load(REF / "tests" / "data" / "meshgrid_regression_case_v1.npz")
    keep = ["nk", "T", "weights", "hamiltonian", "coulomb_q", "hartree_matrix",
            "reference_density", "P0", "electrondensity0", "max_iter", "comm_tol",
            "P_expected", "F_expected", "E_expected", "mu_expected", "k_expected",
            "hist_E_expected", "hist_dC_expected"]
    np.savez_compressed(HERE / "meshgrid_scf_v1.npz", **{k: d[k] for k in keep})
    np.savez_compressed(HERE / "kernel_args_ref.npz", **_ref_cases())
    np.savez_compressed(HERE / "superlattice_ref.npz", **_superlattice_case())
    np.savez_compressed(HERE / "symmetry_ref.npz", **_symmetry_cases())
    print("wrote", HERE / "meshgrid_scf_v1.npz", HERE / "kernel_args_ref.npz", HERE / "superlattice_ref.npz",
          HERE / "symmetry_ref.npz")


if __name__ == "__main__":
    main()
