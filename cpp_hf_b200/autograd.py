"""Differentiable Fock-build API on the B200 library (torch.autograd.Function).

The reference's ``build_fock``, ``hf_energy``, ``occupation_entropy`` and
``free_energy`` (cpp_hf ``fock.py:16-124``) and ``density_from_fock``
(``solver_scf.hpp:96-154``) compute values only.  These wrappers keep their
argument names and results and add backward passes written as CUDA kernels of
``libcpphf_b200.so``:

* exchange: the adjoint of P -> Sigma = -IFFT2[FFT2(P) VR] is the same FFT
  convolution with conj(VR) (``cpphf_exchange_adjoint``); dL/dVR is
  -(1/nk) conj(FFT2(P - refP)) FFT2(dL/dSigma) (``cpphf_exchange_vr_grad``);
* Fock assembly F = herm(h + Sigma + H): ``cpphf_fock_backward_prep``; the
  Hartree and contact terms act on the (nb, nb) mean density and are
  differentiated with small torch ops;
* energy / entropy: ``cpphf_hf_energy[_backward]``,
  ``cpphf_occupation_entropy[_backward]`` (Kahan-compensated deterministic
  reductions);
* density_from_fock: the eigh + Fermi-Dirac adjoint through the occupation
  derivatives with the electron count held fixed
  (``cpphf_density_from_fock_backward``); the forward keeps the per-k
  eigenvectors (not FFT intermediates) for the backward pass.

Tensors are complex128 / float64 CUDA tensors.  ``free_energy_at_convergence``
differentiates a converged direct-minimisation solve with respect to model
parameters: at the minimum the free energy is stationary in (Q, p) at fixed
electron count, so dOmega*/dtheta = dOmega/dtheta at the converged density.
"""

from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from ._lib import check
from ._native import _DeviceKernel, _dev, _lib_handle, _ptr, _stream, _ws

__all__ = [
    "exchange",
    "vr_from_coulomb",
    "build_fock",
    "hf_energy",
    "occupation_entropy",
    "free_energy",
    "density_from_fock",
    "free_energy_at_convergence",
    "solve_model",
    "free_energy_of",
]


def _c(x):
    return x.to(device=_dev(), dtype=torch.complex128).contiguous()


def _f(x):
    return x.to(device=_dev(), dtype=torch.float64).contiguous()


def _herm(X):
    return 0.5 * (X + X.conj().transpose(-1, -2))


# ---------------------------------------------------------------------------
# exchange
# ---------------------------------------------------------------------------

class _Exchange(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, VR):
        lib = _lib_handle()
        nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[2]
        dv = VR.shape[2]
        Sigma = torch.empty_like(P)
        check(lib.cpphf_exchange(_ptr(P), None, _ptr(VR), _ptr(Sigma), nk1, nk2, nb, dv, 0, 0, 64, None, 0,
                                 _stream()), "exchange")
        ctx.save_for_backward(P, VR)
        return Sigma

    @staticmethod
    def backward(ctx, gS):
        P, VR = ctx.saved_tensors
        gS = gS.contiguous()
        lib = _lib_handle()
        nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[2]
        dv = VR.shape[2]
        gP = gVR = None
        if ctx.needs_input_grad[0]:
            gP = torch.empty_like(P)
            check(lib.cpphf_exchange_adjoint(_ptr(gS), _ptr(VR), _ptr(gP), nk1, nk2, nb, dv, _stream()),
                  "exchange adjoint")
        if ctx.needs_input_grad[1]:
            gVR = torch.empty_like(VR)
            ws = _ws(lib.cpphf_exchange_vr_grad_workspace_bytes(nk1, nk2, nb))
            check(lib.cpphf_exchange_vr_grad(_ptr(P), None, _ptr(gS), _ptr(gVR), nk1, nk2, nb, dv, _ptr(ws),
                                             ws.numel(), _stream()), "exchange VR gradient")
        return gP, gVR


def exchange(P, VR):
    """Sigma = -IFFT2[FFT2(P) . VR] (selfenergy_fft with the prephased VR, no ifftshift)."""
    P = _c(P)
    VR = _c(VR)
    if P.dim() != 4 or VR.dim() != 4:
        raise ValueError("P must be (nk1,nk2,nb,nb) and VR (nk1,nk2,dv,dv)")
    return _Exchange.apply(P, VR)


def vr_from_coulomb(Vq, weights):
    """VR = FFT2(w Vq) exp(2 pi i (j s0/n0 + l s1/n1)) with s = n // 2 (problem.py:84-104).

    A one-time setup transform (torch.fft), differentiable in Vq and weights.
    """
    Vq = Vq.to(device=_dev())
    w = _f(weights)
    n0, n1 = w.shape
    X = (w[..., None, None] * Vq).to(torch.complex128)
    VR = torch.fft.fftn(X, dim=(0, 1))
    j = torch.arange(n0, device=_dev(), dtype=torch.float64)
    l = torch.arange(n1, device=_dev(), dtype=torch.float64)
    ph = torch.exp(2j * math.pi * (j[:, None] * (n0 // 2) / n0 + l[None, :] * (n1 // 2) / n1))
    return (VR * ph[..., None, None]).contiguous()


# ---------------------------------------------------------------------------
# build_fock
# ---------------------------------------------------------------------------

def _contact_sigma(rho_bar, cg, cOi, cOj):
    """sum_t g_t [Oi_t tr(Oj_t rho) - Oi_t rho Oj_t]  (fock.py:71-81)."""
    tr = torch.einsum("tij,ji->t", cOj, rho_bar)
    sh = torch.einsum("t,tij->ij", cg.to(tr.dtype) * tr, cOi)
    sf = torch.einsum("t,tij->ij", (-cg).to(rho_bar.dtype), cOi @ rho_bar @ cOj)
    return sh + sf


class _BuildFock(torch.autograd.Function):
    """(P, h, VR, refP, HH) -> (Sigma, Hdiag, F) through cpphf_build_fock."""

    @staticmethod
    def forward(ctx, P, h, VR, refP, HH, meta):
        lib = _lib_handle()
        args, has_refP, include_hartree, include_exchange, cg, cOi, cOj, w2d = meta
        dk = _DeviceKernel(args)
        nk1, nk2, nb = dk.shape
        Sigma = torch.empty_like(P)
        F = torch.empty_like(P)
        hd = torch.zeros(nb, dtype=torch.float64, device=_dev())
        ws = _ws(lib.cpphf_build_fock_workspace_bytes(dk.ref()))
        check(lib.cpphf_build_fock(dk.ref(), _ptr(P), _ptr(Sigma), _ptr(F), _ptr(hd), None, None, _ptr(ws),
                                   ws.numel(), _stream()), "build_fock")
        ctx.meta = meta
        ctx.save_for_backward(P, VR, refP, HH)
        return Sigma, hd, F

    @staticmethod
    def backward(ctx, gSigma, ghd, gF):
        P, VR, refP, HH = ctx.saved_tensors
        args, has_refP, include_hartree, include_exchange, cg, cOi, cOj, w2d = ctx.meta
        lib = _lib_handle()
        nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[2]
        nk = nk1 * nk2
        gS = torch.empty_like(P)
        gh = torch.empty_like(P)
        check(lib.cpphf_fock_backward_prep(_ptr(gSigma.contiguous()) if gSigma is not None else None,
                                           _ptr(gF.contiguous()) if gF is not None else None, _ptr(gS), _ptr(gh),
                                           nk, nb, _stream()), "fock backward")
        dP = P - refP if has_refP else P
        gdP = torch.zeros_like(P)
        if include_exchange:
            check(lib.cpphf_exchange_adjoint(_ptr(gS), _ptr(VR), _ptr(gdP), nk1, nk2, nb, VR.shape[2], _stream()),
                  "exchange adjoint")
        w = w2d.reshape(nk1, nk2)
        gHH = None
        if include_hartree:
            # F gets diag(hd); hd = HH n, n_b = sum_k w_k Re dP_k,bb
            g_hd = torch.diagonal(gh, dim1=-2, dim2=-1).real.sum(dim=(0, 1))
            if ghd is not None:
                g_hd = g_hd + ghd
            g_n = HH.transpose(0, 1) @ g_hd
            idx = torch.arange(nb, device=P.device)
            gdP[..., idx, idx] += (w[..., None] * g_n[None, None, :]).to(gdP.dtype)
            n_vec = (w[..., None] * torch.diagonal(dP, dim1=-2, dim2=-1).real).sum(dim=(0, 1))
            gHH = torch.outer(g_hd, n_vec)
        if cg is not None:
            rho_bar = torch.einsum("ij,ijab->ab", w.to(P.dtype), dP)
            _, vjp = torch.func.vjp(lambda r: _contact_sigma(r, cg, cOi, cOj), rho_bar)
            (g_rho,) = vjp(gS.sum(dim=(0, 1)))
            gdP = gdP + w[..., None, None] * g_rho
        gVR = None
        if ctx.needs_input_grad[2] and include_exchange:
            gVR = torch.empty_like(VR)
            ws = _ws(lib.cpphf_exchange_vr_grad_workspace_bytes(nk1, nk2, nb))
            check(lib.cpphf_exchange_vr_grad(_ptr(P), _ptr(refP) if has_refP else None, _ptr(gS), _ptr(gVR), nk1,
                                             nk2, nb, VR.shape[2], _ptr(ws), ws.numel(), _stream()),
                  "exchange VR gradient")
        g_ref = -gdP if (has_refP and ctx.needs_input_grad[3]) else None
        return gdP, gh, gVR, g_ref, gHH, None


def build_fock(P, *, h, VR, refP=None, HH=None, w2d, include_exchange=True, include_hartree=False,
               exchange_hermitian_channel_packing=False, contact_g=None, contact_Oi=None, contact_Oj=None,
               project_fn=None):
    """``(Sigma, H, F)`` of cpp_hf ``fock.build_fock`` (fock.py:16-88), differentiable in P, h, VR, refP, HH.

    H is ``diag(HH n)[None, None]`` with Hartree, else zeros shaped like h (as the
    reference).  ``exchange_hermitian_channel_packing`` only selects a faster
    forward in the reference and does not change the result; the differentiable
    path always runs the full channel set.  ``project_fn`` is not differentiable
    and is rejected.
    """
    if project_fn is not None:
        raise NotImplementedError("project_fn is not differentiable; apply it outside build_fock")
    P = _c(P)
    h = _c(h)
    VR = _c(VR)
    nk1, nk2, nb = h.shape[0], h.shape[1], h.shape[2]
    w2d = _f(w2d)
    has_refP = refP is not None and refP.numel() > 0
    refP_t = _c(refP) if has_refP else torch.zeros(1, dtype=torch.complex128, device=_dev())
    HH_t = _f(HH) if HH is not None else torch.zeros((nb, nb), dtype=torch.float64, device=_dev())
    contact = contact_g is not None and contact_Oi is not None and contact_Oj is not None
    cg = _f(contact_g) if contact else None
    cOi = _c(contact_Oi) if contact else None
    cOj = _c(contact_Oj) if contact else None
    if include_hartree and not has_refP:
        raise ValueError("include_hartree=True requires reference_density (refP)")
    args = {
        "h": h.detach(), "VR": VR.detach(), "refP": refP_t.detach() if has_refP else np.empty((0,), np.complex128),
        "has_refP": has_refP, "w2d": w2d, "HH": HH_t.detach(),
        "contact_g": cg.detach() if contact else np.zeros((1,)),
        "contact_Oi": cOi.detach() if contact else np.zeros((1, nb, nb), np.complex128),
        "contact_Oj": cOj.detach() if contact else np.zeros((1, nb, nb), np.complex128),
        "weight_sum": float(w2d.sum()), "T": 1.0, "include_hartree": bool(include_hartree),
        "include_exchange": bool(include_exchange), "exchange_hcp": False,
    }
    meta = (args, has_refP, bool(include_hartree), bool(include_exchange), cg, cOi, cOj, w2d.reshape(-1))
    Sigma, hd, F = _BuildFock.apply(P, h, VR, refP_t, HH_t, meta)
    if include_hartree:
        H = torch.diag_embed(hd.to(torch.complex128))[None, None]
    else:
        H = torch.zeros_like(h)
    return Sigma, H, F


# ---------------------------------------------------------------------------
# energies
# ---------------------------------------------------------------------------

class _HfEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, h, Sigma, H, refP, w, H_per_k, has_refP):
        lib = _lib_handle()
        nk = P.shape[0] * P.shape[1]
        nb = P.shape[2]
        E = torch.zeros((), dtype=torch.float64, device=_dev())
        ws = _ws(lib.cpphf_reduce_workspace_bytes())
        check(lib.cpphf_hf_energy(_ptr(h), _ptr(Sigma), _ptr(H), int(H_per_k), _ptr(P),
                                  _ptr(refP) if has_refP else None, _ptr(w), nk, nb, _ptr(E), _ptr(ws), ws.numel(),
                                  _stream()), "hf_energy")
        ctx.save_for_backward(P, h, Sigma, H, refP, w)
        ctx.flags = (H_per_k, has_refP)
        return E

    @staticmethod
    def backward(ctx, gE):
        P, h, Sigma, H, refP, w = ctx.saved_tensors
        H_per_k, has_refP = ctx.flags
        lib = _lib_handle()
        nk = P.shape[0] * P.shape[1]
        nb = P.shape[2]
        need = ctx.needs_input_grad
        gP = torch.empty_like(P) if need[0] else None
        gh = torch.empty_like(h) if need[1] else None
        gSig = torch.empty_like(Sigma) if need[2] else None
        gH = torch.empty_like(H) if need[3] else None
        gref = torch.empty_like(P) if (need[4] and has_refP) else None
        ge = gE.to(torch.float64).reshape(1).contiguous()
        check(lib.cpphf_hf_energy_backward(_ptr(h), _ptr(Sigma), _ptr(H), int(H_per_k), _ptr(P),
                                           _ptr(refP) if has_refP else None, _ptr(w), _ptr(ge), nk, nb, _ptr(gP),
                                           _ptr(gh), _ptr(gSig), _ptr(gH), _ptr(gref), _stream()),
              "hf_energy backward")
        return gP, gh, gSig, gH, gref, None, None, None


def hf_energy(P, *, h, Sigma, H, weights_b, refP=None):
    """E = sum_k w_k Tr[h P] + 1/2 sum_k w_k Tr[(Sigma + H)(P - refP)] (fock.py:91-107)."""
    P = _c(P)
    h = _c(h)
    Sigma = _c(Sigma)
    nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[2]
    H = _c(H)
    if tuple(H.shape) == (nk1, nk2, nb, nb):
        H_per_k = 1
    elif H.numel() == nb * nb:
        H_per_k = 0
        H = H.reshape(nb, nb)
    else:
        raise ValueError("H must be (nk1,nk2,nb,nb) or broadcastable (1,1,nb,nb)")
    w = _f(weights_b).reshape(nk1, nk2, -1)[..., 0].contiguous()
    has_refP = refP is not None and refP.numel() > 0
    refP_t = _c(refP) if has_refP else torch.zeros(1, dtype=torch.complex128, device=_dev())
    return _HfEnergy.apply(P, h, Sigma, H, refP_t, w, H_per_k, has_refP)


class _Entropy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p, wn):
        lib = _lib_handle()
        nb = p.shape[-1]
        nk = p.numel() // nb
        S = torch.zeros((), dtype=torch.float64, device=_dev())
        ws = _ws(lib.cpphf_reduce_workspace_bytes())
        check(lib.cpphf_occupation_entropy(_ptr(p), _ptr(wn), nk, nb, _ptr(S), _ptr(ws), ws.numel(), _stream()),
              "occupation_entropy")
        ctx.save_for_backward(p, wn)
        return S

    @staticmethod
    def backward(ctx, gS):
        p, wn = ctx.saved_tensors
        lib = _lib_handle()
        nb = p.shape[-1]
        nk = p.numel() // nb
        gp = None
        if ctx.needs_input_grad[0]:
            gp = torch.empty_like(p)
            g = gS.to(torch.float64).reshape(1).contiguous()
            check(lib.cpphf_occupation_entropy_backward(_ptr(p), _ptr(wn), _ptr(g), nk, nb, _ptr(gp), _stream()),
                  "occupation_entropy backward")
        return gp, None


def occupation_entropy(p, w_norm):
    """S = -sum w_norm [p ln p + (1 - p) ln(1 - p)], p clipped to [1e-14, 1 - 1e-14] (fock.py:110-113)."""
    p = _f(p)
    wn = _f(w_norm).reshape(-1)
    if wn.numel() * p.shape[-1] != p.numel():
        raise ValueError("w_norm must have one entry per k-point of p")
    return _Entropy.apply(p, wn)


def free_energy(E, p, w_norm, T):
    """Omega = E - max(T, 1e-14) S(p) (fock.py:118-124)."""
    T_val = max(float(T), 1e-14)
    return E - T_val * occupation_entropy(p, w_norm)


# ---------------------------------------------------------------------------
# density_from_fock
# ---------------------------------------------------------------------------

class _DensityFromFock(torch.autograd.Function):
    @staticmethod
    def forward(ctx, F, w, n_e, T):
        lib = _lib_handle()
        nk1, nk2, nb = F.shape[0], F.shape[1], F.shape[2]
        P = torch.empty_like(F)
        V = torch.empty_like(F)
        eps = torch.empty((nk1, nk2, nb), dtype=torch.float64, device=_dev())
        mu = torch.zeros(1, dtype=torch.float64, device=_dev())
        ws = _ws(lib.cpphf_density_from_fock_workspace_bytes(nk1 * nk2, nb))
        check(lib.cpphf_density_from_fock(_ptr(F), _ptr(w), nk1, nk2, nb, float(n_e), float(T), 0.0, _ptr(P),
                                          _ptr(eps), _ptr(V), _ptr(mu), _ptr(ws), ws.numel(), _stream()),
              "density_from_fock")
        ctx.save_for_backward(V, eps, mu, w)
        ctx.T = float(T)
        ctx.mark_non_differentiable(eps, mu)
        return P, eps, mu

    @staticmethod
    def backward(ctx, gP, geps, gmu):
        V, eps, mu, w = ctx.saved_tensors
        lib = _lib_handle()
        nk1, nk2, nb = V.shape[0], V.shape[1], V.shape[2]
        gF = torch.empty_like(V)
        ws = _ws(lib.cpphf_density_from_fock_backward_workspace_bytes())
        # the occupations use expit(-(eps - mu)/(T + 1e-12)) (fermidirac_scalar)
        check(lib.cpphf_density_from_fock_backward(_ptr(V), _ptr(eps), _ptr(mu), ctx.T + 1.0e-12, _ptr(w),
                                                   _ptr(gP.contiguous()), _ptr(gF), nk1 * nk2, nb, _ptr(ws),
                                                   ws.numel(), _stream()), "density_from_fock backward")
        return gF, None, None, None


def density_from_fock(F, weights, n_e, T):
    """(P, eps, mu) of density_from_fock (solver_scf.hpp:96-154, no level shift), differentiable in F.

    The electron count n_e is held fixed: mu moves with F.  eps and mu carry no gradient.
    """
    F = _c(F)
    w = _f(weights).reshape(F.shape[0], F.shape[1]).contiguous()
    if not (float(T) > 0.0):
        raise ValueError("density_from_fock needs T > 0 for a differentiable occupation")
    return _DensityFromFock.apply(F, w, float(n_e), float(T))


# ---------------------------------------------------------------------------
# gradient of the converged free energy
# ---------------------------------------------------------------------------

def _model_kernel_args(m):
    """kernel_args dict (device tensors, exchange only) of a model dict."""
    h = _c(m["h"])
    VR = vr_from_coulomb(m["Vq"], m["weights"])
    w = _f(m["weights"])
    nb = h.shape[2]
    return {
        "h": h, "VR": VR, "refP": np.empty((0,), np.complex128), "has_refP": False, "w2d": w,
        "HH": np.zeros((nb, nb)), "contact_g": np.zeros((1,)),
        "contact_Oi": np.zeros((1, nb, nb), np.complex128), "contact_Oj": np.zeros((1, nb, nb), np.complex128),
        "weight_sum": float(w.sum()), "T": float(m["T"]), "include_hartree": False, "include_exchange": True,
        "exchange_hcp": False,
    }


def solve_model(model, theta, *, method="scf", P0=None, solve_kwargs=None):
    """Converge the model at theta with the library's solve_scf (linear mixing) or solve (direct
    minimisation); returns dict(P, p, iterations, converged, residual) with device tensors.

    At the self-consistent density the occupations are the eigenvalues of P, so
    p is read from eigh(P) for the SCF route.
    """
    from . import _native

    with torch.no_grad():
        m = model(theta.detach().to(device=_dev(), dtype=torch.float64))
        args = _model_kernel_args(m)
        h = args["h"]
        nk1, nk2, nb = h.shape[0], h.shape[1], h.shape[2]
        P0_t = torch.zeros_like(h) if P0 is None else _c(P0)
        n_e = float(m["n_e"])
        if method == "scf":
            kw = dict(max_iter=2000, tol=1e-12, mixing=0.5)
            kw.update(solve_kwargs or {})
            res = _native.solve_scf(args, P0_t, n_e, kw["max_iter"], kw["tol"], kw["tol"], kw["mixing"], 0.0, None,
                                    [], "linear", 6, 2, 1.0, 0.0, False, True)
            # The SCF's chemical potential comes from 30 bisection steps, so its
            # electron count is off by up to ~1e-7, enough to swamp a 1e-5 finite
            # difference.  Re-occupy the final Fock eigenbasis at the mu that
            # holds n_e to machine precision (the in-loop Newton solver).
            F = res[1]
            eps, V = _native.eigh_batched(F)
            w = args["w2d"]
            wsum = float(w.sum())
            lib = _lib_handle()
            mu0 = torch.tensor([float(res[3])], dtype=torch.float64, device=_dev())
            mu = torch.zeros(1, dtype=torch.float64, device=_dev())
            wn = (w / wsum).reshape(-1).contiguous()
            ws = _ws(lib.cpphf_mu_workspace_bytes(nk1 * nk2, nb))
            check(lib.cpphf_solve_mu_inloop(_ptr(eps), _ptr(wn), nk1 * nk2, nb, n_e / wsum, _ptr(mu0), float(m["T"]),
                                            25, _ptr(mu), _ptr(ws), ws.numel(), _stream()), "mu polish")
            p = torch.sigmoid((mu - eps) / max(float(m["T"]), 1e-12))
            P = (V * p[..., None, :].to(V.dtype)) @ V.conj().transpose(-1, -2)
            P = 0.5 * (P + P.conj().transpose(-1, -2))
            return {"P": P.contiguous(), "p": p, "iterations": res[4], "converged": res[5],
                    "residual": float(max(res[7][-1], res[8][-1])) if res[4] else math.inf}
        if method != "dm":
            raise ValueError("method must be 'scf' or 'dm'")
        kw = dict(max_iter=3000, tol_E=1e-13, tol_grad=1e-8)
        kw.update(solve_kwargs or {})
        empty = torch.empty((0, nk1, nk2, nb, nb), dtype=torch.complex128, device=_dev())
        res = _native.solve_dm(args, P0_t, n_e, kw["max_iter"], kw["tol_E"], kw["tol_grad"], 0.6, 0.5, 1e-3, 8, 10,
                               5, 25, 0, 0.5, 20, empty, 0.0, 1.0, [], None, False, True, False)
        return {"P": res[2], "p": res[1], "iterations": res[6], "converged": res[7],
                "residual": float(res[9][-1]) if res[6] else math.inf}


def free_energy_of(model, theta, P, p):
    """Omega(theta) = E[P; h(theta), V(theta)] - T S(p) at a fixed density (differentiable in theta)."""
    m = model(theta)
    VR = vr_from_coulomb(m["Vq"], m["weights"])
    w = _f(m["weights"])
    Sigma, H, F = build_fock(P, h=m["h"], VR=VR, w2d=w, include_exchange=True)
    E = hf_energy(P, h=m["h"], Sigma=Sigma, H=H, weights_b=w[..., None, None])
    wn = (w / w.sum()).reshape(-1)
    return free_energy(E, p, wn, float(m["T"]))


def free_energy_at_convergence(model, theta, *, method="scf", P0=None, solve_kwargs=None):
    """(Omega*, dOmega*/dtheta, info) for a model (h, Vq) = model(theta).

    ``model(theta)`` returns a dict with torch tensors ``h`` (nk1,nk2,nb,nb),
    ``Vq`` (nk1,nk2,dv,dv), ``weights`` (nk1,nk2) and floats ``T``, ``n_e``,
    built from ``theta`` with differentiable torch ops (exchange only, no
    Hartree).  The model is converged with ``solve_model`` (``method`` "scf":
    solve_scf with linear mixing to residuals 1e-12; "dm": direct
    minimisation); at the converged density the free energy is stationary in
    the density at fixed electron count, so dOmega*/dtheta is dOmega/dtheta at
    that density, evaluated through the differentiable build_fock / hf_energy /
    free_energy.  ``info`` is the solve_model dict.
    """
    theta = theta.detach().to(device=_dev(), dtype=torch.float64).requires_grad_(True)
    info = solve_model(model, theta, method=method, P0=P0, solve_kwargs=solve_kwargs)
    Omega = free_energy_of(model, theta, info["P"], info["p"])
    (g,) = torch.autograd.grad(Omega, theta)
    return float(Omega.detach()), g.detach(), info
