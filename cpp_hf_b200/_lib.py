"""ctypes binding of ``libcpphf_b200.so`` (the C ABI declared in ``include/cpphf_b200.h``).

Loading fails loudly: there is no CPU fallback anywhere in this package.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("CPPHF_B200_LIB", HERE / "libcpphf_b200.so"))

CPPHF_OK = 0
CPPHF_ERR_INVALID = -1
CPPHF_ERR_CUDA = -2
CPPHF_ERR_TIMEOUT = -3
CPPHF_ERR_NONFINITE = -4
CPPHF_ERR_UNSUPPORTED = -5

i64 = C.c_int64
i32 = C.c_int32
f64 = C.c_double
vp = C.c_void_p
dp = C.POINTER(C.c_double)
sz = C.c_size_t


class Superlattice(C.Structure):
    """``cpphf_superlattice`` (layout index arrays on the host, Coulomb tables on the device)."""

    _fields_ = [
        ("fock_active", i32), ("hartree_active", i32),
        ("n_G", i64), ("dim_orb", i64), ("n_delta", i64), ("N_ext_x", i64), ("N_ext_y", i64),
        ("hartree_degeneracy", f64),
        ("V_lag_fft", vp), ("V_lag_fft_orbital", vp),
        ("g_a_off", C.POINTER(i64)), ("pair_i", C.POINTER(i64)), ("pair_j", C.POINTER(i64)),
        ("pair_start", C.POINTER(i64)), ("pair_to_delta", C.POINTER(i64)),
        ("HH_GG", vp), ("HH_GG_orbital", vp),
    ]


class Kernel(C.Structure):
    """``cpphf_kernel`` (device pointers)."""

    _fields_ = [
        ("nk1", i64), ("nk2", i64), ("nb", i64), ("dv", i64),
        ("include_hartree", i32), ("include_exchange", i32), ("exchange_hcp", i32),
        ("has_refP", i32), ("has_contact", i32), ("n_contact", i32),
        ("exchange_precision", i32), ("hermitian_packing", i32),
        ("T", f64), ("weight_sum", f64),
        ("h", vp), ("VR", vp), ("refP", vp), ("w2d", vp), ("HH", vp),
        ("contact_g", vp), ("contact_Oi", vp), ("contact_Oj", vp),
        ("sl", C.POINTER(Superlattice)),
        ("VR_packed", vp), ("h_packed", vp),
    ]


class DmConfig(C.Structure):
    _fields_ = [
        ("max_iter", i64), ("tol_E", f64), ("tol_grad", f64), ("plateau_window", i64),
        ("denom_scale", f64), ("max_step", f64), ("cg_restart", i64), ("bt_shrink", f64),
        ("bt_max", i64), ("mu_maxiter", i32), ("optimizer", i32),
        ("block_sizes", C.POINTER(i64)), ("n_block_sizes", i64), ("mixed_switch_grad", f64),
        ("graphs", i32), ("project_device", i32),
        ("tr_delta0", f64), ("tr_cg_max", i64), ("deflation_targets", C.c_void_p), ("n_deflation", i64),
        ("deflation_sigma", f64), ("deflation_length", f64),
    ]


class DmResult(C.Structure):
    _fields_ = [("mu", f64), ("energy", f64), ("n_iter", i64), ("converged", i32), ("reserved", i32)]


class ScfConfig(C.Structure):
    _fields_ = [
        ("max_iter", i64), ("density_tol", f64), ("comm_tol", f64), ("mixing", f64),
        ("level_shift", f64), ("acceleration", i32), ("reserved", i32), ("mixed_switch_tol", f64),
        ("diis_size", i32), ("diis_start", i32), ("diis_damping", f64), ("trust_radius", f64),
        ("graphs", i32), ("reserved1", i32),
        ("block_sizes", C.POINTER(i64)), ("n_block_sizes", i64),
    ]


class ScfResult(C.Structure):
    _fields_ = [("energy", f64), ("mu", f64), ("iterations", i64), ("converged", i32), ("reserved", i32)]


PROJECT_FN = C.CFUNCTYPE(C.c_int, vp, vp, i64, i64, i64, vp)


class Symmetry(C.Structure):
    _fields_ = [
        ("unitary_group", vp), ("n_unitary", i64), ("spatial_group", vp), ("n_spatial", i64),
        ("spatial_convention", i32), ("spatial_axes", i32), ("time_reversal_U", vp), ("tr_convention", i32),
        ("tr_axes", i32), ("scratch", vp),
    ]

# name -> (restype, argtypes)
_SIGS = {
    "cpphf_last_error": (C.c_char_p, []),
    "cpphf_version": (C.c_int, []),
    "cpphf_device_error": (C.c_int, [C.c_int]),
    "cpphf_set_barrier_spin_limit": (C.c_int, [C.c_longlong]),
    "cpphf_barrier_spin_limit": (C.c_longlong, []),
    "cpphf_copy_d2h": (C.c_int, [vp, vp, sz, vp]),
    "cpphf_copy_h2d": (C.c_int, [vp, vp, sz, vp]),
    "cpphf_exchange_workspace_bytes": (sz, [i64, i64, i64, C.c_int, C.c_int]),
    "cpphf_exchange": (C.c_int, [vp, vp, vp, vp, i64, i64, i64, i64, C.c_int, C.c_int, C.c_int,
                                 vp, sz, vp]),
    "cpphf_clear_fft_plan_cache": (C.c_int, []),
    "cpphf_eigh_batched": (C.c_int, [vp, vp, vp, i64, i64, vp]),
    "cpphf_eigh_block_sizes": (C.c_int, [vp, vp, vp, i64, i64, C.POINTER(i64), i64, C.c_int, vp]),
    "cpphf_max_offblock_sizes": (C.c_int, [vp, i64, i64, C.POINTER(i64), i64, vp, vp]),
    "cpphf_mu_workspace_bytes": (sz, [i64, i64]),
    "cpphf_find_mu_bisection": (C.c_int, [vp, vp, i64, i64, f64, f64, C.c_int, vp, vp, sz, vp]),
    "cpphf_solve_mu_inloop": (C.c_int, [vp, vp, i64, i64, f64, vp, f64, C.c_int, vp, vp, sz, vp]),
    "cpphf_find_mu_bisection_noalloc": (C.c_int, [vp, vp, i64, i64, f64, f64, C.c_int, vp, vp]),
    "cpphf_build_fock_workspace_bytes": (sz, [C.POINTER(Kernel)]),
    "cpphf_kernel_packed_bytes": (sz, [C.POINTER(Kernel)]),
    "cpphf_kernel_pack": (C.c_int, [C.POINTER(Kernel), vp, vp, vp]),
    "cpphf_build_fock": (C.c_int, [C.POINTER(Kernel), vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "cpphf_cayley_spectral_setup": (C.c_int, [vp, vp, vp, i64, i64, vp]),
    "cpphf_cayley_unitary": (C.c_int, [vp, vp, f64, vp, i64, i64, vp]),
    "cpphf_diag_ufu": (C.c_int, [vp, vp, vp, f64, vp, i64, i64, vp]),
    "cpphf_solve_dm_workspace_bytes": (sz, [C.POINTER(Kernel)]),
    "cpphf_solve_dm_workspace_bytes_cfg": (sz, [C.POINTER(Kernel), C.POINTER(DmConfig)]),
    "cpphf_rtr_joint_hvp_workspace_bytes": (sz, [C.POINTER(Kernel)]),
    "cpphf_rtr_joint_hvp": (C.c_int, [C.POINTER(Kernel), vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "cpphf_deflation_bias_workspace_bytes": (sz, [i64]),
    "cpphf_deflation_bias": (C.c_int, [vp, vp, i64, vp, i64, i64, i64, f64, f64, vp, dp, vp, sz, vp]),
    "cpphf_solve_dm": (C.c_int, [C.POINTER(Kernel), C.POINTER(DmConfig), vp, f64, PROJECT_FN, vp,
                                 vp, vp, vp, vp, dp, dp, C.POINTER(DmResult), vp, sz, vp]),
    "cpphf_superlattice_workspace_bytes": (sz, [i64, i64, i64, i64, i64, C.c_int]),
    "cpphf_superlattice_streamed": (C.c_int, [vp, vp, vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64),
                                              C.POINTER(i64), i64, i64, i64, i64, i64, i64, i64, C.c_int, vp, vp,
                                              sz, vp]),
    "cpphf_density_from_fock_workspace_bytes": (sz, [i64, i64]),
    "cpphf_density_from_fock": (C.c_int, [vp, vp, i64, i64, i64, f64, f64, f64, vp, vp, vp, vp, vp, sz, vp]),
    "cpphf_exchange_adjoint": (C.c_int, [vp, vp, vp, i64, i64, i64, i64, vp]),
    "cpphf_exchange_vr_grad_workspace_bytes": (sz, [i64, i64, i64]),
    "cpphf_exchange_vr_grad": (C.c_int, [vp, vp, vp, vp, i64, i64, i64, i64, vp, sz, vp]),
    "cpphf_fock_backward_prep": (C.c_int, [vp, vp, vp, vp, i64, i64, vp]),
    "cpphf_reduce_workspace_bytes": (sz, []),
    "cpphf_hf_energy": (C.c_int, [vp, vp, vp, C.c_int, vp, vp, vp, i64, i64, vp, vp, sz, vp]),
    "cpphf_hf_energy_backward": (C.c_int, [vp, vp, vp, C.c_int, vp, vp, vp, vp, i64, i64, vp, vp, vp, vp, vp,
                                           vp]),
    "cpphf_occupation_entropy": (C.c_int, [vp, vp, i64, i64, vp, vp, sz, vp]),
    "cpphf_occupation_entropy_backward": (C.c_int, [vp, vp, vp, i64, i64, vp, vp]),
    "cpphf_density_from_fock_backward_workspace_bytes": (sz, []),
    "cpphf_density_from_fock_backward": (C.c_int, [vp, vp, vp, f64, vp, vp, vp, i64, i64, vp, sz, vp]),
    "cpphf_solve_scf_workspace_bytes": (sz, [C.POINTER(Kernel)]),
    "cpphf_solve_scf_workspace_bytes_cfg": (sz, [C.POINTER(Kernel), C.POINTER(ScfConfig)]),
    "cpphf_resample_kgrid_2d": (C.c_int, [vp, vp, i64, i64, i64, vp]),
    "cpphf_symmetry_project": (C.c_int, [C.POINTER(Symmetry), vp, i64, i64, i64, vp]),
    "cpphf_symmetry_project_fn": (C.c_int, [vp, vp, i64, i64, i64, vp]),
    "cpphf_solve_scf": (C.c_int, [C.POINTER(Kernel), C.POINTER(ScfConfig), vp, f64, PROJECT_FN, vp,
                                  vp, vp, dp, dp, dp, C.POINTER(ScfResult), vp, sz, vp]),
}

_lib = None


def load():
    """Load the shared library once (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m cpp_hf_b200.build` "
            "(this package has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names this binding expects the library to export."""
    return sorted(_SIGS)


class NativeError(RuntimeError):
    pass


def check(status: int, what: str = "") -> None:
    """Map a C status to the reference's Python exception types."""
    if status == CPPHF_OK:
        return
    msg = load().cpphf_last_error().decode(errors="replace")
    if status == CPPHF_ERR_INVALID:
        raise ValueError(msg)
    if status == CPPHF_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise NativeError(f"{what}: status {status}: {msg}")


def check_device_error(what: str = "") -> None:
    """Raise if a bounded device wait gave up since the last check.

    Reads and clears the library's device error word (``cpphf_device_error``,
    which synchronises the device); used by the calls that return host results.
    """
    v = load().cpphf_device_error(1)
    if v == 0:
        return
    if v < 0:
        check(v, what)
    kinds = []
    if v & 2:
        kinds.append("a grid barrier")
    if v & 1:
        kinds.append("an asynchronous-copy wait")
    raise NativeError(f"{what}: status {CPPHF_ERR_TIMEOUT}: {' and '.join(kinds) or 'a wait'} on the device gave up "
                      "(bounded wait timeout)")
