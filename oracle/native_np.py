"""CPU oracle: FP64 NumPy restatement of cpp_hf's ``_native`` operator module.

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
path in ``cpp_hf_b200``; it is imported by ``tests/``, by
``__graft_entry__.smoke()`` and by the CPU-baseline leg of ``bench.py`` and by
nothing else.  The product never calls it.

Every public function has the name, positional/keyword signature, return tuple
and error text of the pybind11 binding in ``cpp/cpp_hf_native.cpp`` of
skilledwolf/cpp_hf, and follows the C++ core statement by statement
(``cpp/include/cpp_hf/*.hpp``).  Third-party arithmetic the reference delegates
to is restated with NumPy equivalents:

* FFTW 3.3.10 guru64 batched 2-D DFT (``fft.hpp:25-142``) -> ``numpy.fft`` /
  ``scipy.fft`` (pocketfft) on axes (0, 1); the inverse is normalised by
  1/(nk1*nk2) exactly like ``FftBatched2D::inverse`` (``fft.hpp:96-111``).
* Eigen 3.4.0 ``SelfAdjointEigenSolver`` (``linalg.hpp:39-55``) -> LAPACK
  ``zheevd`` through ``numpy.linalg.eigh`` (ascending eigenvalues).
* Eigen dense products -> ``numpy.matmul``.

Reductions the reference keeps serial (``parallel.hpp:3-10``) are NumPy sums
here; they differ from the serial order only at the 1e-16 relative level.

Pinning: ``oracle/pin_reference_suite.py`` installs this module as
``cpp_hf._native`` and runs the reference's own pytest suite and its stored
meshgrid regression case against it.
"""

from __future__ import annotations

import copy
import math
import os

import numpy as np

try:  # multithreaded pocketfft, standing in for FFTW threads
    import scipy.fft as _sfft

    _WORKERS = int(os.environ.get("CPPHF_ORACLE_WORKERS", str(os.cpu_count() or 1)))

    def _fft2(x):
        return _sfft.fftn(x, axes=(0, 1), workers=_WORKERS)

    def _ifft2(x):
        return _sfft.ifftn(x, axes=(0, 1), workers=_WORKERS)

except Exception:  # pragma: no cover - scipy is present in this image
    def _fft2(x):
        return np.fft.fftn(x, axes=(0, 1))

    def _ifft2(x):
        return np.fft.ifftn(x, axes=(0, 1))


# types.hpp:13-16
TINY_REAL = 1.0e-30
LOGIT_CLIP = 1.0e-6
ENTROPY_CLIP = 1.0e-14
OCC_CLIP = 1.0e-8

__all__ = [
    "selfenergy_fft_full",
    "clear_fft_plan_cache",
    "eigh_batched",
    "eigh_block_sizes",
    "max_offblock_sizes",
    "find_mu_bisection",
    "build_fock_apply",
    "solve_scf",
    "solve_dm",
    "_cayley_spectral_setup",
    "_cayley_unitary_from_spectrum",
    "_diag_UFU_from_spectrum",
    "_rtr_joint_hvp",
    "_deflation_bias",
    "selfenergy_superlattice_streamed",
    "resample_kgrid_2d",
]


def _c128(x):
    return np.ascontiguousarray(np.asarray(x), dtype=np.complex128)


def _f64(x):
    return np.ascontiguousarray(np.asarray(x), dtype=np.float64)


def _adj(X):
    return np.conj(np.swapaxes(X, -1, -2))


def hermitize(M):
    """linalg.hpp:20-34 (per-element 0.5*(a + conj(b)) on i<=j, mirrored)."""
    return 0.5 * (M + _adj(M))


def expit(x):
    """utils.hpp:18-26 stable sigmoid (branch on the sign of x)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    pos = x >= 0.0
    out[pos] = 1.0 / (1.0 + np.exp(-x[pos]))
    e = np.exp(x[~pos])
    out[~pos] = e / (1.0 + e)
    return out


def fermidirac(x, T):
    """utils.hpp:28-30."""
    return expit(-np.asarray(x, dtype=np.float64) / (T + 1.0e-12))


# ---------------------------------------------------------------------------
# Exchange self-energy (selfenergy.hpp)
# ---------------------------------------------------------------------------

def _exchange_full(rho, VR):
    """selfenergy.hpp:60-117: Sigma = -IFFT2[FFT2(rho) * VR], VR (.,.,1,1) or (.,.,nb,nb)."""
    nb = rho.shape[-1]
    dv1, dv2 = VR.shape[-2], VR.shape[-1]
    if not ((dv1 == 1 and dv2 == 1) or (dv1 == nb and dv2 == nb)):
        raise ValueError("VR shape must be (..., 1, 1) or (..., nb, nb).")
    return -_ifft2(_fft2(rho) * VR)


def _exchange_hcp(rho, VR):
    """selfenergy.hpp:123-171: upper-triangle packing, scalar VR, conj mirror."""
    nb = rho.shape[-1]
    ti, tj = np.triu_indices(nb)
    packed = rho[..., ti, tj]
    sig = -_ifft2(_fft2(packed) * VR[..., 0, 0][..., None])
    out = np.empty_like(rho)
    out[..., ti, tj] = sig
    off = ti != tj
    out[..., tj[off], ti[off]] = np.conj(sig[..., off])
    return out


def _ifftshift_2d(x):
    """selfenergy.hpp:174-190 (out[i,j] = in[(i+n0/2)%n0, (j+n1/2)%n1])."""
    return np.fft.ifftshift(x, axes=(0, 1))


def selfenergy_fft_full(VR, P, apply_ifftshift=True, hermitian_channel_packing=False):
    """cpp_hf_native.cpp:246-278."""
    VR = _c128(VR)
    P = _c128(P)
    if P.ndim != 4:
        raise ValueError("P must be (nk1,nk2,nb,nb)")
    if VR.ndim != 4:
        raise ValueError("VR must be (nk1,nk2,dv1,dv2)")
    if hermitian_channel_packing:
        if VR.shape[2] != 1 or VR.shape[3] != 1:
            raise ValueError("hermitian_channel_packing requires VR with shape (...,1,1)")
        sigma = _exchange_hcp(P, VR)
    else:
        sigma = _exchange_full(P, VR)
    if apply_ifftshift:
        sigma = _ifftshift_2d(sigma)
    return np.ascontiguousarray(sigma)


def clear_fft_plan_cache():
    """cpp_hf_native.cpp:280-284 (pocketfft keeps no plans we own)."""
    return None


# ---------------------------------------------------------------------------
# eigh (linalg.hpp)
# ---------------------------------------------------------------------------

def _eigh(M):
    """linalg.hpp:39-66: hermitise, then ascending eigh per matrix."""
    H = hermitize(M)
    w, V = np.linalg.eigh(H)
    return w, V


def eigh_batched(M):
    """cpp_hf_native.cpp:287-312."""
    M = _c128(M)
    if M.ndim < 2:
        raise ValueError("M needs at least 2 dims")
    if M.shape[-1] != M.shape[-2]:
        raise ValueError("M last two dims must be square")
    w, V = _eigh(M)
    return np.ascontiguousarray(w), np.ascontiguousarray(V)


def _eigh_block_sizes(M, sizes, sort):
    """linalg.hpp:72-120."""
    nb = M.shape[-1]
    lead = M.shape[:-2]
    w = np.zeros(lead + (nb,), dtype=np.float64)
    V = np.zeros(lead + (nb, nb), dtype=np.complex128)
    s0 = 0
    for s in sizes:
        sub = M[..., s0:s0 + s, s0:s0 + s]
        ws, Vs = np.linalg.eigh(hermitize(sub))
        w[..., s0:s0 + s] = ws
        V[..., s0:s0 + s, s0:s0 + s] = Vs
        s0 += s
    if sort:
        order = np.argsort(w, axis=-1, kind="stable")
        w = np.take_along_axis(w, order, axis=-1)
        V = np.take_along_axis(V, order[..., None, :], axis=-1)
    return w, V


def eigh_block_sizes(M, sizes, sort=True):
    """cpp_hf_native.cpp:314-343."""
    M = _c128(M)
    if M.ndim < 2:
        raise ValueError("M needs at least 2 dims")
    sizes = [int(s) for s in sizes]
    if sum(sizes) != M.shape[-1]:
        raise ValueError("block sizes must sum to nb")
    w, V = _eigh_block_sizes(M, sizes, bool(sort))
    return np.ascontiguousarray(w), np.ascontiguousarray(V)


def _offblock_mask(nb, sizes):
    mask = np.ones((nb, nb), dtype=bool)
    s0 = 0
    for s in sizes:
        mask[s0:s0 + s, s0:s0 + s] = False
        s0 += s
    return mask


def max_offblock_sizes(M, sizes):
    """linalg.hpp:123-140; cpp_hf_native.cpp:345-358."""
    M = _c128(M)
    nb = M.shape[-1]
    mask = _offblock_mask(nb, [int(s) for s in sizes])
    if not mask.any() or M.size == 0:
        return 0.0
    return float(np.max(np.abs(M[..., mask])))


# ---------------------------------------------------------------------------
# chemical potential (utils.hpp)
# ---------------------------------------------------------------------------

def _find_mu_bisection(eps, weights, n_e, T, maxiter=0):
    """utils.hpp:49-75 (fixed iteration count, count > n_e -> hi)."""
    if maxiter <= 0:
        maxiter = 30
    eps = np.asarray(eps, dtype=np.float64)
    nb = eps.shape[-1]
    eps2 = eps.reshape(-1, nb)
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    Tj = max(T, 1.0e-12)
    emin = float(eps2.min())
    emax = float(eps2.max())
    span = emax - emin + 10.0 * max(Tj, 1.0e-6)
    lo = emin - span
    hi = emax + span
    for _ in range(int(maxiter)):
        mid = 0.5 * (lo + hi)
        count = float(np.sum(w[:, None] * fermidirac(eps2 - mid, Tj)))
        if count > n_e:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def _solve_mu_inloop(eps, w_norm, n_target_norm, mu0, T, maxiter=25):
    """utils.hpp:79-116 (Newton step inside a bisection bracket)."""
    eps = np.asarray(eps, dtype=np.float64)
    nb = eps.shape[-1]
    eps2 = eps.reshape(-1, nb)
    w = np.asarray(w_norm, dtype=np.float64).reshape(-1)[:, None]
    Tj = max(T, 1.0e-12)
    emin = float(eps2.min())
    emax = float(eps2.max())
    lo = emin - 50.0 * Tj
    hi = emax + 50.0 * Tj
    mu = min(max(mu0, lo), hi)
    for _ in range(int(maxiter)):
        p = expit((mu - eps2) / Tj)
        N = float(np.sum(w * p))
        Z = float(np.sum(w * p * (1.0 - p) / Tj))
        g = N - n_target_norm
        if g < 0.0:
            lo = mu
        if g > 0.0:
            hi = mu
        Z_safe = max(Z, 1.0e-18)
        mu_new = mu - g / Z_safe
        mu_bis = 0.5 * (lo + hi)
        if mu_new <= lo or mu_new >= hi:
            mu_new = mu_bis
        mu_new = min(max(mu_new, lo), hi)
        if not math.isfinite(mu_new):
            mu_new = mu_bis
        mu = mu_new
    return mu


def find_mu_bisection(bands, weights, n_e, T, maxiter=0):
    """cpp_hf_native.cpp:361-377."""
    bands = _f64(bands)
    weights = _f64(weights)
    return float(_find_mu_bisection(bands, weights, float(n_e), float(T), int(maxiter)))


# ---------------------------------------------------------------------------
# Kernel view (kernel.hpp; cpp_hf_native.cpp:42-213)
# ---------------------------------------------------------------------------

class _Kernel:
    """Mirror of ``HFKernel`` (kernel.hpp:10-84) built from a kernel_args dict."""

    def __init__(self, args):
        h = _c128(args["h"])
        if h.ndim != 4:
            raise ValueError("h must be (nk1,nk2,nb,nb)")
        self.nk1, self.nk2, self.nb = h.shape[0], h.shape[1], h.shape[2]
        if h.shape[3] != self.nb:
            raise ValueError("h last two axes must be square (nb,nb)")
        VR = _c128(args["VR"])
        if VR.ndim != 4:
            raise ValueError("VR must be (nk1,nk2,dv1,dv2)")
        self.dv1, self.dv2 = VR.shape[2], VR.shape[3]
        if not ((self.dv1 == 1 and self.dv2 == 1) or (self.dv1 == self.nb and self.dv2 == self.nb)):
            raise ValueError("VR last two dims must be (1,1) or (nb,nb)")
        self.h = h
        self.VR = VR
        self.include_hartree = bool(args["include_hartree"])
        self.include_exchange = bool(args["include_exchange"])
        self.exchange_hcp = bool(args["exchange_hcp"])
        self.has_refP = bool(args["has_refP"])
        self.T = float(args["T"])
        self.weight_sum = float(args["weight_sum"])
        if self.has_refP:
            refP = _c128(args["refP"])
            if refP.shape != h.shape:
                raise ValueError("refP must match h shape when has_refP is true")
            self.refP = refP
        else:
            self.refP = None
        self.w2d = _f64(args["w2d"]).reshape(self.nk1, self.nk2)
        self.HH = _f64(args["HH"]).reshape(self.nb, self.nb)
        cg = _f64(args["contact_g"])
        if cg.ndim != 1:
            raise ValueError("contact_g must be 1-D")
        self.contact_g = cg
        self.n_contact = cg.shape[0]
        self.contact_Oi = _c128(args["contact_Oi"]).reshape(self.n_contact, self.nb, self.nb)
        self.contact_Oj = _c128(args["contact_Oj"]).reshape(self.n_contact, self.nb, self.nb)

        # superlattice injection (cpp_hf_native.cpp:109-213)
        self.sl_fock = bool(args.get("superlattice_fock_active", False))
        self.sl_hartree = bool(args.get("superlattice_hartree_active", False))
        if self.sl_fock or self.sl_hartree:
            self.hartree_degeneracy = float(args.get("hartree_degeneracy", 1.0))
            self.n_G = int(args["n_G"])
            self.dim_orb = int(args["dim_orb"])
            self.n_delta = int(args["n_delta"])
            self.N_ext_x = int(args["N_ext_x"])
            self.N_ext_y = int(args["N_ext_y"])
            if self.n_G * self.dim_orb != self.nb:
                raise ValueError("superlattice mode requires n_G × dim_orb == nb")
            self.V_lag_fft = _c128(args["V_lag_fft"])
            self.g_a_off = np.ascontiguousarray(args["g_a_off"], dtype=np.int64)
            self.pair_i = np.ascontiguousarray(args["pair_i"], dtype=np.int64)
            self.pair_j = np.ascontiguousarray(args["pair_j"], dtype=np.int64)
            self.pair_start = np.ascontiguousarray(args["pair_start"], dtype=np.int64)
            self.pair_to_delta = np.ascontiguousarray(args["pair_to_delta"], dtype=np.int64)
            if self.V_lag_fft.shape[:2] != (self.N_ext_x, self.N_ext_y):
                raise ValueError("V_lag_fft must have shape (N_ext_x, N_ext_y)")
            if self.g_a_off.shape != (self.n_G, 2):
                raise ValueError("g_a_off must be (n_G, 2)")
            if self.pair_start.shape[0] != self.n_delta + 1:
                raise ValueError("pair_start must have length n_delta + 1")
            if self.pair_i.shape[0] != self.pair_j.shape[0]:
                raise ValueError("pair_i and pair_j must have the same length")
            if self.pair_to_delta.shape != (self.n_G, self.n_G):
                raise ValueError("pair_to_delta must be (n_G, n_G)")
            self.V_lag_fft_orbital = None
            if "V_lag_fft_orbital" in args:
                vo = _c128(args["V_lag_fft_orbital"])
                if vo.shape != (self.N_ext_x, self.N_ext_y, self.dim_orb, self.dim_orb):
                    raise ValueError(
                        "V_lag_fft_orbital must be (N_ext_x, N_ext_y, dim_orb, dim_orb)")
                self.V_lag_fft_orbital = vo
            self.HH_GG = None
            self.HH_GG_orbital = None
            if self.sl_hartree:
                hg = _f64(args["HH_GG"])
                if hg.shape != (self.n_G, self.n_G):
                    raise ValueError("HH_GG must be (n_G, n_G)")
                self.HH_GG = hg
                if "HH_GG_orbital" in args:
                    ho = _f64(args["HH_GG_orbital"])
                    if ho.shape != (self.n_G, self.n_G, self.dim_orb, self.dim_orb):
                        raise ValueError("HH_GG_orbital must be (n_G, n_G, dim_orb, dim_orb)")
                    self.HH_GG_orbital = ho

    def has_contact_terms(self):
        """fock.hpp:25-29."""
        if np.any(self.contact_g != 0.0):
            return True
        return self.n_contact > 1


def _call_project(project_fn, M):
    """cpp_hf_native.cpp:215-238: view in, forcecast C-contiguous complex128 out."""
    out = np.ascontiguousarray(np.asarray(project_fn(M)), dtype=np.complex128)
    if out.ndim != 4 or out.shape != M.shape:
        raise RuntimeError("project_fn returned an array of wrong shape")
    return out.copy()


# ---------------------------------------------------------------------------
# Superlattice streamed Fock (superlattice.hpp)
# ---------------------------------------------------------------------------

def _superlattice_streamed(rho, VR_fft, VR_fft_orbital, g_a_off, pair_i, pair_j,
                           pair_start, n_delta, N_ext_x, N_ext_y, nkx, nky, n_G,
                           dim_orb, hermitian_rho):
    """superlattice.hpp:50-246 (per-ΔG scatter -> FFT conv -> gather)."""
    rho6 = rho.reshape(nkx, nky, n_G, dim_orb, n_G, dim_orb)
    sigma = np.zeros_like(rho6)
    partner = np.full(n_delta, -1, dtype=np.int64)
    if hermitian_rho:
        key_to_ch = {}
        rkeys = []
        for d in range(n_delta):
            a, b = int(pair_start[d]), int(pair_start[d + 1])
            key = tuple(sorted(int(pair_i[p]) * n_G + int(pair_j[p]) for p in range(a, b)))
            rkey = tuple(sorted(int(pair_j[p]) * n_G + int(pair_i[p]) for p in range(a, b)))
            key_to_ch.setdefault(key, d)
            rkeys.append(rkey)
        for d in range(n_delta):
            partner[d] = key_to_ch.get(rkeys[d], -1)
    if VR_fft_orbital is not None:
        VRk = VR_fft_orbital
    else:
        VRk = VR_fft.reshape(N_ext_x, N_ext_y, 1, 1)
    for dg in range(n_delta):
        pr = int(partner[dg])
        has_partner = pr >= 0 and pr != dg
        if has_partner and pr < dg:
            continue
        a, b = int(pair_start[dg]), int(pair_start[dg + 1])
        if a == b:
            continue
        buf = np.zeros((N_ext_x, N_ext_y, dim_orb, dim_orb), dtype=np.complex128)
        for p in range(a, b):
            i, j = int(pair_i[p]), int(pair_j[p])
            ox = nkx * int(g_a_off[i, 0])
            oy = nky * int(g_a_off[i, 1])
            buf[ox:ox + nkx, oy:oy + nky] = rho6[:, :, i, :, j, :]
        if not np.any(buf):
            continue
        buf = _exchange_full(buf, VRk)
        for p in range(a, b):
            i, j = int(pair_i[p]), int(pair_j[p])
            ox = nkx * int(g_a_off[i, 0])
            oy = nky * int(g_a_off[i, 1])
            blk = buf[ox:ox + nkx, oy:oy + nky]
            sigma[:, :, i, :, j, :] = blk
            if has_partner:
                sigma[:, :, j, :, i, :] = np.conj(np.swapaxes(blk, -1, -2))
    return sigma


def selfenergy_superlattice_streamed(rho, VR_fft, g_a_off, pair_i, pair_j, pair_start,
                                     nkx, nky, n_G, dim_orb, N_ext_x, N_ext_y,
                                     VR_fft_orbital=None, hermitian_rho=False):
    """cpp_hf_native.cpp:719-816."""
    rho = _c128(rho)
    VR_fft = _c128(VR_fft)
    g_a_off = np.ascontiguousarray(g_a_off, dtype=np.int64)
    pair_i = np.ascontiguousarray(pair_i, dtype=np.int64)
    pair_j = np.ascontiguousarray(pair_j, dtype=np.int64)
    pair_start = np.ascontiguousarray(pair_start, dtype=np.int64)
    if rho.ndim != 6:
        raise ValueError("rho must be (nkx, nky, n_G, dim_orb, n_G, dim_orb)")
    if VR_fft.ndim != 2:
        raise ValueError("VR_fft must be (N_ext_x, N_ext_y)")
    if VR_fft.shape != (N_ext_x, N_ext_y):
        raise ValueError("VR_fft shape does not match (N_ext_x, N_ext_y)")
    if g_a_off.ndim != 2 or g_a_off.shape != (n_G, 2):
        raise ValueError("g_a_off must be (n_G, 2)")
    if pair_start.ndim != 1 or pair_start.shape[0] < 1:
        raise ValueError("pair_start must be 1-D, len >= 1")
    if pair_i.ndim != 1 or pair_j.ndim != 1 or pair_i.shape[0] != pair_j.shape[0]:
        raise ValueError("pair_i and pair_j must be 1-D with the same length")
    vo = None
    if VR_fft_orbital is not None:
        vo = _c128(VR_fft_orbital)
        if vo.ndim != 4 or vo.shape != (N_ext_x, N_ext_y, dim_orb, dim_orb):
            raise ValueError("VR_fft_orbital must be (N_ext_x, N_ext_y, dim_orb, dim_orb)")
    n_delta = pair_start.shape[0] - 1
    out = _superlattice_streamed(rho, VR_fft, vo, g_a_off, pair_i, pair_j, pair_start,
                                 n_delta, int(N_ext_x), int(N_ext_y), int(nkx), int(nky),
                                 int(n_G), int(dim_orb), bool(hermitian_rho))
    return np.ascontiguousarray(out.reshape(rho.shape))


# ---------------------------------------------------------------------------
# Fock assembly and energies (fock.hpp)
# ---------------------------------------------------------------------------

def _sl_hartree_matrix(K, rho):
    """fock.hpp:66-175 (k-independent superlattice Hartree shift)."""
    nb, nG, orb, nd = K.nb, K.n_G, K.dim_orb, K.n_delta
    rho_bar = np.einsum("ij,ijab->ab", K.w2d, rho)
    rb = rho_bar.reshape(nG, orb, nG, orb)
    p2d = K.pair_to_delta
    out = np.zeros((nb, nb), dtype=np.complex128)
    deg = K.hartree_degeneracy
    if K.HH_GG_orbital is None:
        rho_GG = np.einsum("axbx->ab", rb)
        rho_for_delta = np.zeros(nd, dtype=np.complex128)
        np.add.at(rho_for_delta, p2d.reshape(-1), rho_GG.reshape(-1))
        s = (deg * K.HH_GG) * rho_for_delta[p2d]
        o6 = out.reshape(nG, orb, nG, orb)
        for xi in range(orb):
            o6[:, xi, :, xi] = s
    else:
        rpd = np.zeros((nd, orb), dtype=np.complex128)
        diag_blocks = np.einsum("agbg->abg", rb)  # (nG, nG, orb)
        np.add.at(rpd, p2d.reshape(-1), diag_blocks.reshape(-1, orb))
        o6 = out.reshape(nG, orb, nG, orb)
        s = np.einsum("abxg,abg->abx", deg * K.HH_GG_orbital, rpd[p2d])
        for al in range(orb):
            o6[:, al, :, al] = s[:, :, al]
    return out


def _build_fock_compact(K, P, project_fn=None):
    """fock.hpp:34-299 -> (Sigma, F, hartree_diag)."""
    nb = K.nb
    need_rho = K.include_exchange or K.sl_hartree
    rho = None
    sl_h = None
    if need_rho:
        rho = P - K.refP if K.has_refP else P.copy()
        if K.include_hartree and K.sl_hartree:
            sl_h = _sl_hartree_matrix(K, rho)
    if K.include_exchange:
        if K.sl_fock:
            Sigma = _superlattice_streamed(
                rho, K.V_lag_fft, K.V_lag_fft_orbital, K.g_a_off, K.pair_i, K.pair_j,
                K.pair_start, K.n_delta, K.N_ext_x, K.N_ext_y, K.nk1, K.nk2, K.n_G,
                K.dim_orb, True).reshape(P.shape)
        elif K.exchange_hcp and K.dv1 == 1 and K.dv2 == 1:
            Sigma = _exchange_hcp(rho, K.VR)
        else:
            Sigma = _exchange_full(rho, K.VR)
    else:
        Sigma = np.zeros_like(P)
    if sl_h is not None:
        Sigma = Sigma + sl_h
    hd = np.zeros(nb, dtype=np.float64)
    if K.include_hartree and not K.sl_hartree:
        diag = np.real(np.diagonal(P, axis1=-2, axis2=-1))
        if K.has_refP:
            diag = diag - np.real(np.diagonal(K.refP, axis1=-2, axis2=-1))
        n_vec = np.einsum("ij,ija->a", K.w2d, diag)
        hd = K.HH @ n_vec
    if K.has_contact_terms():
        dP = P - K.refP if K.has_refP else P
        rho_bar = np.einsum("ij,ijab->ab", K.w2d, dP)
        SC = np.zeros((nb, nb), dtype=np.complex128)
        for t in range(K.n_contact):
            g = K.contact_g[t]
            if g == 0.0:
                continue
            Oi, Oj = K.contact_Oi[t], K.contact_Oj[t]
            tr = np.sum(Oj * rho_bar.T)
            SC += Oi * tr * g + (-g) * (Oi @ rho_bar @ Oj)
        Sigma = Sigma + SC
    F = K.h + Sigma
    if K.include_hartree:
        idx = np.arange(nb)
        F = F.copy()
        F[..., idx, idx] += hd
    F = hermitize(F)
    if project_fn is not None:
        F = hermitize(_call_project(project_fn, F))
    return np.ascontiguousarray(Sigma), np.ascontiguousarray(F), hd


def _hf_energy_hd(K, P, Sigma, hd):
    """fock.hpp:355-383: sum_k w_k [Re Tr(h P) + Re Tr(inter (P - refP))]."""
    dP = P - K.refP if K.has_refP else P
    inter = 0.5 * Sigma
    if K.include_hartree:
        idx = np.arange(K.nb)
        inter = inter.copy()
        inter[..., idx, idx] += 0.5 * hd
    one = np.real(np.einsum("...ij,...ji->...", K.h, P))
    two = np.real(np.einsum("...ij,...ji->...", inter, dP))
    return float(np.sum(K.w2d * (one + two)))


def build_fock_apply(kernel_args, P, project_fn):
    """cpp_hf_native.cpp:380-415 -> (Sigma, H, F, E)."""
    K = _Kernel(kernel_args)
    P = _c128(P)
    pf = None if project_fn is None else project_fn
    Sigma, F, hd = _build_fock_compact(K, P, pf)
    Hh = np.zeros_like(P)
    if K.include_hartree:
        idx = np.arange(K.nb)
        Hh[..., idx, idx] = hd
    # fock.hpp:324-351 (hf_energy with a dense H) == the compact form here.
    dP = P - K.refP if K.has_refP else P
    one = np.real(np.einsum("...ij,...ji->...", K.h, P))
    two = np.real(np.einsum("...ij,...ji->...", 0.5 * (Sigma + Hh), dP))
    E = float(np.sum(K.w2d * (one + two)))
    return Sigma, Hh, F, E


def occupation_entropy(p, w_norm):
    """fock.hpp:385-401."""
    pv = np.clip(np.asarray(p, dtype=np.float64), ENTROPY_CLIP, 1.0 - ENTROPY_CLIP)
    s = pv * np.log(pv) + (1.0 - pv) * np.log1p(-pv)
    return float(-np.sum(np.asarray(w_norm)[..., None] * s))


def free_energy_value(E, p, w_norm, T):
    """fock.hpp:403-407."""
    return float(E - max(T, 1.0e-14) * occupation_entropy(p, w_norm))


# ---------------------------------------------------------------------------
# Direct minimisation (solver_dm.hpp)
# ---------------------------------------------------------------------------

def _cayley_factor(lam, tau):
    """solver_dm.hpp:251-255."""
    arg = 0.5 * tau * np.asarray(lam, dtype=np.float64)
    iexp = 1j * arg
    return (1.0 + iexp) / (1.0 - iexp)


def _cayley_setup(d):
    """solver_dm.hpp:206-222: eigh of hermitised i*d."""
    iA = 1j * d
    w, V = np.linalg.eigh(hermitize(iA))
    return V, w


def _cayley_unitary(V, lam, tau):
    """solver_dm.hpp:258-272."""
    c = _cayley_factor(lam, tau)
    return (V * c[..., None, :]) @ _adj(V)


def _diag_UFU(V, Fe, lam, tau):
    """solver_dm.hpp:277-303."""
    c = _cayley_factor(lam, tau)
    M = np.conj(c)[..., :, None] * Fe * c[..., None, :]
    A = V @ M
    return np.real(np.sum(A * np.conj(V), axis=-1))


def _ip_matrix(X, Y, w):
    """solver_dm.hpp:163-177."""
    per_k = np.real(np.sum(np.conj(X) * Y, axis=(-2, -1)))
    return float(np.sum(w * per_k))


def _ip_vec(x, y, w):
    """solver_dm.hpp:179-191."""
    return float(np.sum(w * np.sum(x * y, axis=-1)))


def _frozen_free_energy(eps, p, w, T):
    """solver_dm.hpp:346-365 (and 367-388 with p - tau*d_p already applied)."""
    pv = np.clip(p, OCC_CLIP, 1.0 - OCC_CLIP)
    E = float(np.sum(w[..., None] * pv * eps))
    S = -float(np.sum(w[..., None] * (pv * np.log(pv) + (1.0 - pv) * np.log1p(-pv))))
    return E - max(T, 1.0e-14) * S


def _block_sizes_enabled(sizes, nb):
    """solver_dm.hpp:80-90."""
    if not sizes:
        return False
    for s in sizes:
        if s == 0:
            raise ValueError("block_sizes entries must be positive.")
    if sum(sizes) != nb:
        raise ValueError("block_sizes must sum to nb.")
    return len(sizes) > 1


def _block_structure_ok(M, nb, sizes):
    """solver_dm.hpp:92-98."""
    mask = _offblock_mask(nb, sizes)
    scale = float(np.max(np.abs(M))) if M.size else 0.0
    off = float(np.max(np.abs(M[..., mask]))) if mask.any() and M.size else 0.0
    return off <= 1.0e-10 + 1.0e-10 * scale


def _block_problem_invariant(K, project_fn, sizes):
    """solver_dm.hpp:100-115."""
    if project_fn is not None:
        return False
    nb = K.nb
    if not _block_structure_ok(K.h, nb, sizes):
        return False
    if K.has_refP and not _block_structure_ok(K.refP, nb, sizes):
        return False
    for t in range(K.n_contact):
        if K.contact_g[t] == 0.0:
            continue
        if not _block_structure_ok(K.contact_Oi[t], nb, sizes):
            return False
        if not _block_structure_ok(K.contact_Oj[t], nb, sizes):
            return False
    return True


def _cayley_setup_blocks(d, sizes):
    """solver_dm.hpp:224-248."""
    nb = d.shape[-1]
    V = np.zeros_like(d)
    lam = np.zeros(d.shape[:-1], dtype=np.float64)
    iA = 1j * d
    s0 = 0
    for s in sizes:
        sub = iA[..., s0:s0 + s, s0:s0 + s]
        w, Vs = np.linalg.eigh(hermitize(sub))
        lam[..., s0:s0 + s] = w
        V[..., s0:s0 + s, s0:s0 + s] = Vs
        s0 += s
    return V, lam


def _solve_dm(K, P0, n_e, cfg, project_fn=None):
    """solver_dm.hpp:392-653 (optimizer == 0, preconditioned Riemannian CG)."""
    nk1, nk2, nb = K.nk1, K.nk2, K.nb
    sizes = list(cfg["block_sizes"])
    block_cfg = _block_sizes_enabled(sizes, nb)
    use_block = block_cfg and _block_problem_invariant(K, project_fn, sizes)

    ws = max(K.weight_sum, TINY_REAL)
    w = K.w2d / ws
    n_t = n_e / ws
    T_r = max(K.T, 1.0e-12)
    max_iter = int(cfg["max_iter"])
    mu_maxiter = int(cfg["mu_maxiter"])

    hist_E = np.zeros(max_iter, dtype=np.float64)
    hist_g = np.zeros(max_iter, dtype=np.float64)

    def eigh_F(F):
        if use_block:
            return _eigh_block_sizes(F, sizes, False)
        return _eigh(F)

    def project(M):
        if project_fn is not None:
            return _call_project(project_fn, M)
        return M

    # init (solver_dm.hpp:436-459)
    P_cur = hermitize(P0)
    Sigma, F, hd = _build_fock_compact(K, P_cur, None)
    if use_block and not _block_structure_ok(F, nb, sizes):
        use_block = False
    eps, Q = eigh_F(F)
    mu0 = _solve_mu_inloop(eps, w, n_t, 0.0, T_r, mu_maxiter)
    p = expit((mu0 - eps) / T_r)
    mu = mu0

    G_Q_prev = np.zeros_like(Q)
    g_p_prev = np.zeros_like(p)
    d_Q_prev = np.zeros_like(Q)
    d_p_prev = np.zeros_like(p)
    grad_norm = math.inf
    E_prev = math.inf
    dE = math.inf
    k = 0
    tol_E = float(cfg["tol_E"])
    tol_grad = float(cfg["tol_grad"])
    pw = int(cfg["plateau_window"])
    while k < max_iter:
        if pw > 0 and k > pw:
            e_now = hist_E[k - 1]
            e_past = hist_E[k - 1 - pw]
            e_nc = (e_past - e_now) > tol_E
        else:
            e_nc = dE > tol_E
        g_nc = (tol_grad > 0.0) and (grad_norm > tol_grad)
        if not (e_nc or g_nc):
            break
        # 1. density, Fock, energy, Ft
        P_cur = (Q * p[..., None, :]) @ _adj(Q)
        P_cur = hermitize(project(P_cur))
        Sigma, F, hd = _build_fock_compact(K, P_cur, None)
        E = _hf_energy_hd(K, P_cur, Sigma, hd)
        Ft = _adj(Q) @ F @ Q
        eps = np.real(np.diagonal(Ft, axis1=-2, axis2=-1)).copy()
        # 2. gradient (solver_dm.hpp:142-160, 504-511)
        dp_ij = p[..., None, :] - p[..., :, None]  # p_j - p_i
        A = dp_ij * Ft
        G_Q = 0.5 * (A - _adj(A))
        idx = np.arange(nb)
        G_Q[..., idx, idx] = 0.0
        pv = np.clip(p, LOGIT_CLIP, 1.0 - LOGIT_CLIP)
        g_p = eps + T_r * (np.log(pv) - np.log1p(-pv)) - mu
        grad_norm = math.sqrt(max(0.0, _ip_matrix(G_Q, G_Q, w)))
        # 3. precondition (solver_dm.hpp:513-541)
        eps_sq = float(np.sum(eps * eps))
        eps_scale = math.sqrt(eps_sq / max(eps.size, 1) + TINY_REAL)
        lam_pc = max(T_r, float(cfg["denom_scale"]) * eps_scale)
        gap = eps[..., :, None] - eps[..., None, :]
        d_Q = G_Q / np.sqrt(gap * gap + lam_pc * lam_pc)
        ps = np.clip(p, OCC_CLIP, 1.0 - OCC_CLIP)
        curv = T_r / (ps * (1.0 - ps))
        h_p = g_p / curv
        # 4. PR+ (solver_dm.hpp:543-559)
        pr_num = (_ip_matrix(G_Q, d_Q, w) - _ip_matrix(G_Q_prev, d_Q, w)
                  + _ip_vec(g_p, h_p, w) - _ip_vec(g_p_prev, h_p, w))
        pr_den = _ip_matrix(G_Q_prev, G_Q_prev, w) + _ip_vec(g_p_prev, g_p_prev, w)
        beta = max(0.0, pr_num / pr_den) if pr_den > TINY_REAL else 0.0
        beta = min(beta, 5.0)
        cg_restart = int(cfg["cg_restart"])
        if k == 0 or (cg_restart > 0 and k % cg_restart == 0):
            beta = 0.0
        d_Q = d_Q + beta * d_Q_prev
        d_p = h_p + beta * d_p_prev
        # 5. line search (solver_dm.hpp:561-589)
        if use_block:
            V_d, lam_d = _cayley_setup_blocks(d_Q, sizes)
        else:
            V_d, lam_d = _cayley_setup(d_Q)
        Fe = _adj(V_d) @ Ft @ V_d
        dQn = math.sqrt(max(0.0, _ip_matrix(d_Q, d_Q, w)))
        tau0 = min(1.0, float(cfg["max_step"]) / max(dQn, TINY_REAL))
        Om0 = _frozen_free_energy(eps, p, w, T_r)
        tau = tau0
        acc = False
        for _bt in range(int(cfg["bt_max"])):
            ew = _diag_UFU(V_d, Fe, lam_d, tau)
            Om = _frozen_free_energy(ew, p - tau * d_p, w, T_r)
            if Om < Om0:
                acc = True
                break
            tau *= float(cfg["bt_shrink"])
        if not acc:
            tau = tau0 * float(cfg["bt_shrink"]) ** float(cfg["bt_max"])
        # 6. retraction
        Q = Q @ _cayley_unitary(V_d, lam_d, tau)
        ew = _diag_UFU(V_d, Fe, lam_d, tau)
        mu_new = _solve_mu_inloop(ew, w, n_t, mu, T_r, mu_maxiter)
        p = expit((mu_new - ew) / T_r)
        mu = mu_new
        # 7. record
        hist_E[k] = E
        hist_g[k] = grad_norm
        dE = abs(E - E_prev)
        d_Q_prev, d_p_prev, G_Q_prev, g_p_prev = d_Q, d_p, G_Q, g_p
        E_prev = E
        k += 1

    # finalize (solver_dm.hpp:615-652)
    P_cur = hermitize(project((Q * p[..., None, :]) @ _adj(Q)))
    Sigma, F, hd = _build_fock_compact(K, P_cur, None)
    Ft = _adj(Q) @ F @ Q
    ew, Vf = eigh_F(Ft)
    Q = Q @ Vf
    mu = _solve_mu_inloop(ew, w, n_t, mu, T_r, mu_maxiter)
    p = expit((mu - ew) / T_r)
    P_cur = hermitize(project((Q * p[..., None, :]) @ _adj(Q)))
    Sigma, F, hd = _build_fock_compact(K, P_cur, None)
    E_fin = _hf_energy_hd(K, P_cur, Sigma, hd)
    return dict(Q=Q, p=p, density=P_cur, fock=F, mu=mu, energy=E_fin, n_iter=k,
                converged=k < max_iter, hist_E=hist_E[:k].copy(), hist_grad=hist_g[:k].copy())


# ---------------------------------------------------------------------------
# Trust-region Newton (optimizer == 1) and the deflation bias
# ---------------------------------------------------------------------------


def _fock_response(K, dP):
    """solver_rtr.hpp:31-39: Sigma[dP] = F[dP] - h with the reference density off."""
    Kr = copy.copy(K)
    Kr.has_refP = False
    Kr.refP = None
    _S, F, _hd = _build_fock_compact(Kr, dP, None)
    return F - K.h


def _project_occ(dp, w2d):
    """solver_rtr.hpp:42-50: remove the w2d-weighted mean so sum_k w_k sum_b dp = 0."""
    nb = dp.shape[-1]
    num = float(np.sum(w2d[..., None] * dp))
    den = float(np.sum(w2d)) * nb
    shift = num / den if den > 0.0 else 0.0
    return dp - shift


def _joint_hvp(K, X, dp, Q, p, Ft, T_r, pen_diag=0.0):
    """solver_rtr.hpp:55-111: joint (Q, p) Hessian-vector product (one Fock build)."""
    nb = K.nb
    idx = np.arange(nb)
    pdiff = p[..., None, :] - p[..., :, None]  # p_j - p_i
    M = X * pdiff
    M[..., idx, idx] = dp
    dP = hermitize(Q @ M @ _adj(Q))
    R = _fock_response(K, dP)
    if pen_diag != 0.0:
        R = R + pen_diag * dP
    St = _adj(Q) @ R @ Q
    A = Ft @ X - X @ Ft + St
    ddiff = dp[..., None, :] - dp[..., :, None]
    C = ddiff * Ft + pdiff * A
    HX = 0.5 * (C - _adj(C))
    HX[..., idx, idx] = 0.0
    pc = np.clip(p, OCC_CLIP, 1.0 - OCC_CLIP)
    Hp = np.real(np.diagonal(A, axis1=-2, axis2=-1)) + T_r / (pc * (1.0 - pc)) * dp
    return HX, _project_occ(Hp, K.w2d)


def _deflation_terms(P, targets, w2d, sigma, length):
    """solver_rtr.hpp:124-157 -> (Phi, S_pen, diag_coeff); a no-op without targets or sigma."""
    S_pen = np.zeros_like(P)
    if targets is None or len(targets) == 0 or sigma == 0.0:
        return 0.0, S_pen, 0.0
    inv2L2 = 1.0 / (2.0 * float(length) * float(length))
    Phi = 0.0
    diag = 0.0
    for T in targets:
        D = P - T
        d2 = float(np.sum(w2d * np.sum(np.abs(D) ** 2, axis=(-2, -1))))
        phi = float(sigma) * math.exp(-d2 * inv2L2)
        phip = -phi * inv2L2
        Phi += phi
        diag += phip
        S_pen = S_pen + (2.0 * phip) * D
    return Phi, S_pen, 2.0 * diag


def _solve_rtr(K, P0, n_e, cfg, project_fn=None):
    """solver_rtr.hpp:163-459 (optimizer == 1): Steihaug truncated CG on the joint
    (Q, p) quadratic model inside a trust region, Cayley retraction with tau = -1."""
    nk1, nk2, nb = K.nk1, K.nk2, K.nb
    T_r = max(K.T, 1.0e-12)
    tol_g = cfg["tol_grad"] if cfg["tol_grad"] > 0.0 else 1.0e-6
    ws = max(K.weight_sum, TINY_REAL)
    w_norm = K.w2d / ws
    n_t = n_e / ws
    w2d = K.w2d
    max_iter = int(cfg["max_iter"])
    mu_maxiter = int(cfg["mu_maxiter"])
    idx = np.arange(nb)
    targets = cfg["deflation_targets"]
    n_defl = 0 if targets is None else int(targets.shape[0])
    d_sigma = float(cfg["deflation_sigma"])
    d_len = max(float(cfg["deflation_length"]), 1.0e-12)
    defl_on = n_defl > 0 and d_sigma > 0.0

    def jip(aX, ap, bX, bp):
        return _ip_matrix(aX, bX, 1.0) + _ip_vec(ap, bp, w2d)

    def jfro(aX, ap):
        return math.sqrt(max(0.0, jip(aX, ap, aX, ap)))

    def prec(aX, ap, lam, eps, p):
        gap = eps[..., :, None] - eps[..., None, :]
        oX = aX / np.sqrt(gap * gap + lam * lam)
        pc = np.clip(p, OCC_CLIP, 1.0 - OCC_CLIP)
        return oX, _project_occ(ap * pc * (1.0 - pc) / T_r, w2d)

    def project(M):
        return _call_project(project_fn, M) if project_fn is not None else M

    # init (solver_rtr.hpp:251-262)
    P_cur = hermitize(P0)
    _S, F, _hd = _build_fock_compact(K, P_cur, None)
    eps, Q = _eigh(F)
    mu = _solve_mu_inloop(eps, w_norm, n_t, 0.0, T_r, mu_maxiter)
    p = expit((mu - eps) / T_r)

    def eval_state(Qs, ps):
        # solver_rtr.hpp:264-285
        P = hermitize(project((Qs * ps[..., None, :]) @ _adj(Qs)))
        Sigma, F, hd = _build_fock_compact(K, P, None)
        E = _hf_energy_hd(K, P, Sigma, hd)
        pen = 0.0
        if defl_on:
            Phi, S_pen, pen = _deflation_terms(P, targets, w2d, d_sigma, d_len)
            E += Phi
            F = F + S_pen
        Ft = _adj(Qs) @ F @ Qs
        eps = np.real(np.diagonal(Ft, axis1=-2, axis2=-1)).copy()
        A = (ps[..., None, :] - ps[..., :, None]) * Ft
        G = 0.5 * (A - _adj(A))
        G[..., idx, idx] = 0.0
        return E, Ft, eps, G, pen

    E, Ft, eps, G, pen = eval_state(Q, p)
    Delta = float(cfg["tr_delta0"])
    hist_E = np.zeros(max_iter, dtype=np.float64)
    hist_g = np.zeros(max_iter, dtype=np.float64)
    k = 0
    converged = False
    while k < max_iter:
        grad_norm = math.sqrt(max(0.0, _ip_matrix(G, G, w_norm)))
        hist_E[k] = E
        hist_g[k] = grad_norm
        if grad_norm < tol_g:
            converged = True
            k += 1
            break
        eps_sq = float(np.sum(eps * eps))
        lam = max(T_r, float(cfg["denom_scale"]) * math.sqrt(eps_sq / max(eps.size, 1) + TINY_REAL))
        # Steihaug truncated CG (solver_rtr.hpp:304-364)
        vX = np.zeros_like(G)
        vp = np.zeros_like(p)
        HvX = np.zeros_like(G)
        Hvp = np.zeros_like(p)
        rX = -G
        rp = np.zeros_like(p)
        zX, zp = prec(rX, rp, lam, eps, p)
        dX, dp = zX, zp
        rz = jip(rX, rp, zX, zp)
        for _cg in range(int(cfg["tr_cg_max"])):
            HDX, HDp = _joint_hvp(K, dX, dp, Q, p, Ft, T_r, pen)
            dHd = jip(dX, dp, HDX, HDp)
            dd = jip(dX, dp, dX, dp)

            def to_boundary(vX, vp, HvX, Hvp):
                a = dd
                b = 2.0 * jip(vX, vp, dX, dp)
                c = jfro(vX, vp)
                cc = c * c - Delta * Delta
                t = (-b + math.sqrt(max(b * b - 4.0 * a * cc, 0.0))) / (2.0 * a + 1e-30)
                return vX + t * dX, vp + t * dp, HvX + t * HDX, Hvp + t * HDp

            if dHd <= 1e-14 * dd:
                vX, vp, HvX, Hvp = to_boundary(vX, vp, HvX, Hvp)
                break
            alpha = rz / dHd
            s2 = float(np.sum(np.abs(vX + alpha * dX) ** 2))
            s2 += float(np.sum(w2d * np.sum((vp + alpha * dp) ** 2, axis=-1)))
            if math.sqrt(max(0.0, s2)) >= Delta:
                vX, vp, HvX, Hvp = to_boundary(vX, vp, HvX, Hvp)
                break
            vX = vX + alpha * dX
            HvX = HvX + alpha * HDX
            rX = rX - alpha * HDX
            vp = vp + alpha * dp
            Hvp = Hvp + alpha * HDp
            rp = rp - alpha * HDp
            rn = math.sqrt(max(0.0, jip(rX, rp, rX, rp)))
            if rn < 0.05 * grad_norm:
                break
            zX, zp = prec(rX, rp, lam, eps, p)
            rz_new = jip(rX, rp, zX, zp)
            beta = rz_new / rz
            dX = zX + beta * dX
            dp = zp + beta * dp
            rz = rz_new
        # predicted reduction in energy units (solver_rtr.hpp:366-378)
        gv = _ip_matrix(G, vX, w2d)
        vHv = _ip_matrix(vX, HvX, w2d) + _ip_vec(vp, Hvp, w2d)
        pred = -(gv + 0.5 * vHv)
        if Delta < 1e-10:
            break
        # retraction Q <- Q Cayley(tau = -1, vX), trial occupations (solver_rtr.hpp:380-396)
        Vd, lamd = _cayley_setup(vX)
        U = _cayley_unitary(Vd, lamd, -1.0)
        Qt = Q @ U
        eps_t = np.real(np.diagonal(_adj(U) @ Ft @ U, axis1=-2, axis2=-1)).copy()
        mu_t = _solve_mu_inloop(eps_t, w_norm, n_t, mu, T_r, mu_maxiter)
        p_t = expit((mu_t - eps_t) / T_r)
        E_t, Ft_t, eps_tr, G_t, pen_t = eval_state(Qt, p_t)
        grad_t = math.sqrt(max(0.0, _ip_matrix(G_t, G_t, w_norm)))
        # acceptance and radius update (solver_rtr.hpp:406-420)
        noise = 1e-12 * max(abs(E), 1.0)
        if pred <= noise:
            accept = (grad_t <= grad_norm) and (E_t <= E + noise)
            if not accept:
                Delta *= 0.5
        else:
            ratio = (E - E_t) / pred
            if ratio < 0.25:
                Delta *= 0.25
            elif ratio > 0.75 and jfro(vX, vp) > 0.9 * Delta:
                Delta = min(2.0 * Delta, 5.0)
            accept = ratio > 0.1
        if accept:
            Q, p, E, mu = Qt, p_t, E_t, mu_t
            Ft, eps, G, pen = Ft_t, eps_tr, G_t, pen_t
        k += 1

    # finalize (solver_rtr.hpp:437-443)
    P_cur = hermitize(project((Q * p[..., None, :]) @ _adj(Q)))
    Sigma, F, hd = _build_fock_compact(K, P_cur, None)
    E_fin = _hf_energy_hd(K, P_cur, Sigma, hd)
    return dict(Q=Q, p=p, density=P_cur, fock=F, mu=mu, energy=E_fin, n_iter=k,
                converged=converged, hist_E=hist_E[:k].copy(), hist_grad=hist_g[:k].copy())


def solve_dm(kernel_args, P0, n_e, max_iter, tol_E, tol_grad, max_step, bt_shrink,
             denom_scale, bt_max, cg_restart, plateau_window, mu_maxiter, optimizer,
             tr_delta0, tr_cg_max, deflation_targets, deflation_sigma, deflation_length,
             block_sizes, project_fn, return_Q, return_density, return_fock):
    """cpp_hf_native.cpp:488-582 (optimizer 0: solver_dm.hpp, 1: solver_rtr.hpp)."""
    K = _Kernel(kernel_args)
    P0 = _c128(P0)
    cfg = dict(max_iter=int(max_iter), tol_E=float(tol_E), tol_grad=float(tol_grad),
               max_step=float(max_step), bt_shrink=float(bt_shrink),
               denom_scale=float(denom_scale), bt_max=int(bt_max),
               cg_restart=int(cg_restart), plateau_window=int(plateau_window),
               mu_maxiter=int(mu_maxiter), block_sizes=[int(s) for s in block_sizes])
    if int(optimizer) == 1:
        # cpp_hf_native.cpp:533-547: targets of shape (n, nk1, nk2, nb, nb), n > 0
        # solver_rtr.hpp:196-205: the size is checked only when deflation is on
        targets = None
        if deflation_targets is not None and float(deflation_sigma) > 0.0:
            t = _c128(deflation_targets)
            if t.ndim == 5 and t.shape[0] > 0:
                if t.size < t.shape[0] * P0.size:
                    raise ValueError("deflation_targets buffer smaller than n_deflation * nk * nb * nb.")
                targets = t.reshape((t.shape[0],) + P0.shape)
        cfg.update(tr_delta0=float(tr_delta0), tr_cg_max=int(tr_cg_max), deflation_targets=targets,
                   deflation_sigma=float(deflation_sigma), deflation_length=float(deflation_length))
        r = _solve_rtr(K, P0, float(n_e), cfg, project_fn)
    else:
        r = _solve_dm(K, P0, float(n_e), cfg, project_fn)
    shape = P0.shape
    return (
        np.ascontiguousarray(r["Q"]).reshape(shape) if return_Q else None,
        np.ascontiguousarray(r["p"]).reshape(shape[:3]),
        np.ascontiguousarray(r["density"]).reshape(shape) if return_density else None,
        np.ascontiguousarray(r["fock"]).reshape(shape) if return_fock else None,
        float(r["mu"]), float(r["energy"]), int(r["n_iter"]), bool(r["converged"]),
        r["hist_E"], r["hist_grad"],
    )


def _cayley_spectral_setup(d):
    """cpp_hf_native.cpp:585-609."""
    d = _c128(d)
    if d.ndim < 2:
        raise ValueError("d needs at least 2 dims")
    if d.shape[-1] != d.shape[-2]:
        raise ValueError("d last two dims must match")
    V, lam = _cayley_setup(d)
    return np.ascontiguousarray(V), np.ascontiguousarray(lam)


def _cayley_unitary_from_spectrum(V, lam, tau):
    """cpp_hf_native.cpp:611-630."""
    V = _c128(V)
    lam = _f64(lam)
    if V.ndim < 2:
        raise ValueError("V needs at least 2 dims")
    return np.ascontiguousarray(_cayley_unitary(V, lam, float(tau)))


def _diag_UFU_from_spectrum(V, Ft_eig, lam, tau):
    """cpp_hf_native.cpp:632-651."""
    V = _c128(V)
    Ft_eig = _c128(Ft_eig)
    lam = _f64(lam)
    if V.ndim < 2:
        raise ValueError("V needs at least 2 dims")
    return np.ascontiguousarray(_diag_UFU(V, Ft_eig, lam, float(tau)))


def _rtr_joint_hvp(kernel_args, X, dp, Q, p, Ft):
    """cpp_hf_native.cpp:654-694: joint (Q, p) Hessian-vector product -> (HX, Hp)."""
    K = _Kernel(kernel_args)
    shape = (K.nk1, K.nk2, K.nb, K.nb)
    X = _c128(X).reshape(shape)
    Q = _c128(Q).reshape(shape)
    Ft = _c128(Ft).reshape(shape)
    dp = _f64(dp).reshape(shape[:3])
    p = _f64(p).reshape(shape[:3])
    HX, Hp = _joint_hvp(K, X, dp, Q, p, Ft, max(K.T, 1.0e-12))
    return np.ascontiguousarray(HX), np.ascontiguousarray(Hp)


def _deflation_bias(P, targets, w2d, sigma, length):
    """cpp_hf_native.cpp:697-716 -> (Phi, S_pen, diag_coeff)."""
    P = _c128(P)
    t = _c128(targets)
    w2d = _f64(w2d).reshape(P.shape[:2])
    tl = t.reshape((t.shape[0],) + P.shape) if (t.ndim == 5 and t.shape[0] > 0) else None
    Phi, S_pen, diag = _deflation_terms(P, tl, w2d, float(sigma), float(length))
    return float(Phi), np.ascontiguousarray(S_pen), float(diag)


# ---------------------------------------------------------------------------
# SCF (solver_scf.hpp)
# ---------------------------------------------------------------------------

def _wnorm(M, w2d, weight_sum):
    """solver_scf.hpp:64-75."""
    per_k = np.sum(np.real(M) ** 2 + np.imag(M) ** 2, axis=(-2, -1))
    return math.sqrt(float(np.sum(w2d * per_k)) / max(weight_sum, 1.0e-30))


def _density_from_fock(F, w2d, n_e, T, level_shift, block_sizes):
    """solver_scf.hpp:96-154 -> (P_new, mu)."""
    nb = F.shape[-1]
    used = False
    if block_sizes:
        if sum(block_sizes) == nb and len(block_sizes) > 1:
            scale = float(np.max(np.abs(F)))
            mask = _offblock_mask(nb, block_sizes)
            off = float(np.max(np.abs(F[..., mask]))) if mask.any() else 0.0
            if off <= 1.0e-10 + 1.0e-10 * scale:
                eps, V = _eigh_block_sizes(F, block_sizes, False)
                used = True
    if not used:
        eps, V = _eigh(F)
    mu_raw = _find_mu_bisection(eps, w2d, n_e, T)
    if level_shift != 0.0:
        occ_raw = fermidirac(eps - mu_raw, T)
        shifted = eps + level_shift * (1.0 - occ_raw)
    else:
        shifted = eps
    mu = _find_mu_bisection(shifted, w2d, n_e, T)
    occ = fermidirac(shifted - mu, T)
    P = (V * occ[..., None, :]) @ _adj(V)
    return hermitize(P), mu


def _solve_scf(K, P0, n_e, cfg, project_fn=None):
    """solver_scf.hpp:156-444."""
    max_iter = int(cfg["max_iter"])
    hist_E = np.zeros(max_iter)
    hist_D = np.zeros(max_iter)
    hist_C = np.zeros(max_iter)
    density = P0.copy()
    acc = cfg["acceleration"]
    use_diis = acc == "diis"
    use_oda = acc == "oda"
    if acc != "linear" and not use_diis and not use_oda:
        raise ValueError("SCFConfig.acceleration must be 'linear', 'diis', or 'oda'")
    level_shift = float(cfg["level_shift"])
    sizes = list(cfg["block_sizes"])
    mixing = float(cfg["mixing"])
    state = {}

    def project(M):
        return _call_project(project_fn, M) if project_fn is not None else M

    def build_and_occupy(d):
        d = hermitize(project(d))
        Sigma, F, hd = _build_fock_compact(K, d, project_fn)
        E = _hf_energy_hd(K, d, Sigma, hd)
        P_new, mu = _density_from_fock(F, K.w2d, n_e, K.T, level_shift, sizes)
        P_new = hermitize(project(P_new))
        state["F"] = F
        return d, P_new, E, mu

    diis_F, diis_R = [], []
    E = 0.0
    mu = 0.0
    converged = False
    k = 0
    while k < max_iter and not converged:
        density, P_new, E_it, mu_it = build_and_occupy(density)
        F = state["F"]
        delta = P_new - density
        comm = F @ density - density @ F
        d_res = _wnorm(delta, K.w2d, K.weight_sum)
        c_res = _wnorm(comm, K.w2d, K.weight_sum)
        converged = (d_res <= float(cfg["density_tol"])) and (c_res <= float(cfg["comm_tol"]))
        tr = float(cfg["trust_radius"])
        density_pre = density.copy() if (tr > 0.0 and not converged) else None
        if converged:
            density = P_new
        elif use_diis:
            if len(diis_F) >= int(cfg["diis_size"]):
                diis_F.pop(0)
                diis_R.pop(0)
            diis_F.append(F.copy())
            diis_R.append(comm.copy())
            m = len(diis_F)
            if m >= max(2, int(cfg["diis_start"])):
                B = np.zeros((m + 1, m + 1))
                rhs = np.zeros(m + 1)
                for i in range(m):
                    for j in range(i, m):
                        per_k = np.real(np.sum(np.conj(diis_R[i]) * diis_R[j], axis=(-2, -1)))
                        B[i, j] = float(np.sum(K.w2d * per_k))
                        B[j, i] = B[i, j]
                    B[i, m] = -1.0
                    B[m, i] = -1.0
                rhs[m] = -1.0
                ok = True
                try:
                    sol = np.linalg.solve(B, rhs)
                    # FullPivLU::isInvertible uses a rank threshold; restated with
                    # the matrix rank at LAPACK's default tolerance.
                    ok = np.linalg.matrix_rank(B) == m + 1
                except np.linalg.LinAlgError:
                    ok = False
                    sol = np.full(m + 1, np.nan)
                ok = ok and bool(np.all(np.isfinite(sol[:m])))
                if ok:
                    F_ex = np.zeros_like(F)
                    for i in range(m):
                        F_ex = F_ex + sol[i] * diis_F[i]
                    damp = min(max(float(cfg["diis_damping"]), 0.0), 1.0)
                    if damp < 1.0:
                        F_ex = damp * F_ex + (1.0 - damp) * F
                    F_ex = hermitize(F_ex)
                    P_d, _ = _density_from_fock(F_ex, K.w2d, n_e, K.T, level_shift, sizes)
                    density = hermitize(project(P_d))
                else:
                    density = hermitize(project(density + mixing * delta))
            else:
                density = hermitize(project(density + mixing * delta))
        elif use_oda:
            Sn, Fn, hdn = _build_fock_compact(K, P_new, project_fn)
            E_new = _hf_energy_hd(K, P_new, Sn, hdn)
            c1 = float(np.sum(K.w2d * np.real(np.einsum("...ab,...ba->...", F, delta))))
            c2 = (E_new - E_it) - c1
            if c2 > 1.0e-12:
                lam = min(max(-c1 / (2.0 * c2), 0.0), 1.0)
            elif c1 < 0.0:
                lam = 1.0
            else:
                lam = 0.0
            density = hermitize(project(density + lam * delta))
        else:
            density = hermitize(project(density + mixing * delta))
        if tr > 0.0 and not converged and density_pre is not None:
            diff = density - density_pre
            step = _wnorm(diff, K.w2d, K.weight_sum)
            if step > tr:
                s = tr / step
                density = hermitize(project(density_pre + s * diff))
        hist_E[k] = E_it
        hist_D[k] = d_res
        hist_C[k] = c_res
        E = E_it
        mu = mu_it
        k += 1
    density, _P, E_fin, mu_fin = build_and_occupy(density)
    return dict(density=density, fock=state["F"], energy=E_fin, mu=mu_fin, iterations=k,
                converged=converged, hist_E=hist_E[:k].copy(), hist_D=hist_D[:k].copy(),
                hist_C=hist_C[:k].copy())


def solve_scf(kernel_args, P0, n_e, max_iter, density_tol, comm_tol, mixing, level_shift,
              project_fn, block_sizes, acceleration, diis_size, diis_start, diis_damping,
              trust_radius, return_density, return_fock):
    """cpp_hf_native.cpp:418-485."""
    K = _Kernel(kernel_args)
    P0 = _c128(P0)
    cfg = dict(max_iter=int(max_iter), density_tol=float(density_tol),
               comm_tol=float(comm_tol), mixing=float(mixing),
               level_shift=float(level_shift), block_sizes=[int(s) for s in block_sizes],
               acceleration=str(acceleration), diis_size=int(diis_size),
               diis_start=int(diis_start), diis_damping=float(diis_damping),
               trust_radius=float(trust_radius))
    r = _solve_scf(K, P0, float(n_e), cfg, project_fn)
    return (
        np.ascontiguousarray(r["density"]) if return_density else None,
        np.ascontiguousarray(r["fock"]) if return_fock else None,
        float(r["energy"]), float(r["mu"]), int(r["iterations"]), bool(r["converged"]),
        r["hist_E"], r["hist_D"], r["hist_C"],
    )


# ---------------------------------------------------------------------------
# k-grid resample (utils.hpp:120-176)
# ---------------------------------------------------------------------------

def _resample_axis(x, n_new):
    n_old = x.shape[0]
    if n_old == n_new:
        return x.copy()
    ratio = n_old / n_new
    s_new = n_new // 2
    s_old = n_old // 2
    out = np.empty((n_new,) + x.shape[1:], dtype=np.complex128)
    for j in range(n_new):
        u = (j - s_new) * ratio + s_old
        fu = math.floor(u)
        i0 = int(fu) % n_old
        i1 = (i0 + 1) % n_old
        frac = u - fu
        out[j] = (1.0 - frac) * x[i0] + frac * x[i1]
    return out


def resample_kgrid_2d(values, nk_new):
    """cpp_hf_native.cpp:819-840."""
    x = _c128(values)
    if x.ndim < 2:
        raise ValueError("need >= 2 dims")
    if x.shape[1] != x.shape[0]:
        raise ValueError("First two axes must be square (nk_old, nk_old)")
    nk_new = int(nk_new)
    if x.shape[0] == nk_new:
        return x.copy()
    t = _resample_axis(x, nk_new)
    out = np.swapaxes(_resample_axis(np.swapaxes(t, 0, 1), nk_new), 0, 1)
    return np.ascontiguousarray(out)
