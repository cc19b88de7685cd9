"""GPU: backward passes of the differentiable Fock-build API against central
finite differences (step 1e-5 unless stated), torch.fft references and the
oracle, including the differentiation workload (layered model, 96x96, nb = 8).

Directional checks: for a real loss L and a complex direction D the derivative
d/dt L(x + t D) equals Re sum conj(grad x) D (torch's complex-gradient convention).
"""

from __future__ import annotations

import numpy as np
import pytest

from cpp_hf_b200 import problem, workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

H_FD = 1.0e-5


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def _cplx(rng, shape, herm=False):
    A = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    if herm:
        A = 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))
    return torch.from_numpy(A).to(_dev())


def _real(rng, shape):
    return torch.from_numpy(rng.normal(size=shape)).to(_dev())


def _inner(g, d):
    return float((g.conj() * d).real.sum()) if g.is_complex() else float((g * d).sum())


def _fd(f, x, d, h=H_FD):
    return (float(f(x + h * d)) - float(f(x - h * d))) / (2.0 * h)


def _check_dir(f, x, d, g, rtol=1e-6, atol=1e-10):
    fd = _fd(f, x, d)
    an = _inner(g, d)
    print(f"fd {fd:.12e} autograd {an:.12e} rel {abs(fd - an) / max(abs(fd), 1e-30):.2e}")
    assert abs(fd - an) <= rtol * max(abs(fd), abs(an)) + atol


def _torch_exchange(P, VR):
    """-IFFT2[FFT2(P) VR] with torch.fft (reference for the CUDA exchange)."""
    X = torch.fft.fftn(P, dim=(0, 1))
    return -torch.fft.ifftn(X * VR, dim=(0, 1))


@pytest.mark.parametrize("dv_full", [True, False])
def test_exchange_adjoint_and_vr_grad_match_torch_fft(dv_full):
    from cpp_hf_b200 import autograd as ag

    rng = np.random.default_rng(1)
    n0, n1, nb = 12, 10, 3
    P = _cplx(rng, (n0, n1, nb, nb)).requires_grad_(True)
    VR = _cplx(rng, (n0, n1, nb, nb) if dv_full else (n0, n1, 1, 1)).requires_grad_(True)
    C = _cplx(rng, (n0, n1, nb, nb))
    S = ag.exchange(P, VR)
    np.testing.assert_allclose(S.detach().cpu().numpy(), _torch_exchange(P, VR).detach().cpu().numpy(),
                               rtol=1e-12, atol=1e-12)
    L = (C.conj() * S).real.sum()
    gP, gV = torch.autograd.grad(L, (P, VR))
    P2 = P.detach().clone().requires_grad_(True)
    V2 = VR.detach().clone().requires_grad_(True)
    L2 = (C.conj() * _torch_exchange(P2, V2)).real.sum()
    rP, rV = torch.autograd.grad(L2, (P2, V2))
    np.testing.assert_allclose(gP.cpu().numpy(), rP.cpu().numpy(), rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(gV.cpu().numpy(), rV.cpu().numpy(), rtol=1e-11, atol=1e-11)


def _fock_case(seed, n=8, nb=4):
    rng = np.random.default_rng(seed)
    w = np.full((n, n), 1.0 / (n * n))
    h = rng.normal(size=(n, n, nb, nb)) + 1j * rng.normal(size=(n, n, nb, nb))
    h = 0.5 * (h + np.conj(np.swapaxes(h, -1, -2)))
    Vq = rng.uniform(0.1, 1.0, size=(n, n, nb, nb))
    Vq = 0.5 * (Vq + np.swapaxes(Vq, -1, -2))
    refP = rng.normal(size=(n, n, nb, nb)) * 0.1 + 0j
    HH = rng.normal(size=(nb, nb))
    Oi = rng.normal(size=(2, nb, nb)) + 1j * rng.normal(size=(2, nb, nb))
    Oj = rng.normal(size=(2, nb, nb)) + 1j * rng.normal(size=(2, nb, nb))
    contact = [(0.3, Oi[0], Oj[0]), (-0.2, Oi[1], Oj[1])]
    args = problem.kernel_args(w, h, Vq, 0.1, include_hartree=True, include_exchange=True, reference_density=refP,
                               hartree_matrix=HH, contact_terms=contact)
    return rng, args


def test_build_fock_forward_matches_native_and_backward_matches_fd(native):
    from cpp_hf_b200 import autograd as ag

    rng, a = _fock_case(3)
    n, nb = a["h"].shape[0], a["h"].shape[2]
    P = _cplx(rng, (n, n, nb, nb), herm=True)
    h = torch.from_numpy(a["h"]).to(_dev())
    VR = torch.from_numpy(a["VR"]).to(_dev())
    refP = torch.from_numpy(a["refP"]).to(_dev())
    HH = torch.from_numpy(a["HH"]).to(_dev())
    cg = torch.from_numpy(a["contact_g"]).to(_dev())
    cOi = torch.from_numpy(a["contact_Oi"]).to(_dev())
    cOj = torch.from_numpy(a["contact_Oj"]).to(_dev())
    w = torch.from_numpy(a["w2d"]).to(_dev())
    kw = dict(w2d=w, include_exchange=True, include_hartree=True, contact_g=cg, contact_Oi=cOi, contact_Oj=cOj)
    S, H, F = ag.build_fock(P, h=h, VR=VR, refP=refP, HH=HH, **kw)
    S0, H0, F0, _E0 = native.build_fock_apply(a, P, None)
    np.testing.assert_allclose(F.detach().cpu().numpy(), F0.cpu().numpy(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(S.detach().cpu().numpy(), S0.cpu().numpy(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(H.detach().cpu().numpy()[0, 0], H0.cpu().numpy()[0, 0], rtol=1e-12, atol=1e-12)
    CF, CS = _cplx(rng, F.shape), _cplx(rng, S.shape)
    CH = _cplx(rng, (1, 1, nb, nb))

    def loss(P_, h_, VR_, refP_, HH_):
        S_, H_, F_ = ag.build_fock(P_, h=h_, VR=VR_, refP=refP_, HH=HH_, **kw)
        return ((CF.conj() * F_).real.sum() + (CS.conj() * S_).real.sum() + (CH.conj() * H_).real.sum())

    xs = [t.detach().clone().requires_grad_(True) for t in (P, h, VR, refP, HH)]
    grads = torch.autograd.grad(loss(*xs), xs)
    for idx, name in enumerate(["P", "h", "VR", "refP", "HH"]):
        x0 = xs[idx].detach()
        d = _cplx(rng, x0.shape) if x0.is_complex() else _real(rng, x0.shape)

        def f(x, idx=idx):
            args = [t.detach() for t in xs]
            args[idx] = x
            with torch.no_grad():
                return loss(*args)

        print(name, end=": ")
        _check_dir(f, x0, d, grads[idx])


def test_hf_energy_and_free_energy_backward(native, oracle):
    from cpp_hf_b200 import autograd as ag

    rng, a = _fock_case(5)
    n, nb = a["h"].shape[0], a["h"].shape[2]
    P = _cplx(rng, (n, n, nb, nb), herm=True)
    h = torch.from_numpy(a["h"]).to(_dev())
    S = _cplx(rng, (n, n, nb, nb), herm=True)
    H = _cplx(rng, (1, 1, nb, nb), herm=True)
    refP = torch.from_numpy(a["refP"]).to(_dev())
    w = torch.from_numpy(a["w2d"]).to(_dev())
    wb = w[..., None, None]
    E = ag.hf_energy(P, h=h, Sigma=S, H=H, weights_b=wb, refP=refP)
    # reference formula (fock.py:91-107) in numpy
    Pn, hn, Sn, Hn, Rn = (t.cpu().numpy() for t in (P, h, S, H, refP))
    dP = Pn - Rn
    ref = np.sum(np.real(a["w2d"] * np.einsum("...ij,...ji->...", hn, Pn)
                         + 0.5 * a["w2d"] * (np.einsum("...ij,...ji->...", Sn, dP)
                                             + np.einsum("...ij,...ji->...", np.broadcast_to(Hn, dP.shape), dP))))
    assert abs(float(E) - ref) < 1e-12 * max(1.0, abs(ref))
    p = torch.from_numpy(rng.uniform(0.05, 0.95, size=(n, n, nb))).to(_dev())
    p[0, 0, 0] = 0.0  # clipped entry: no gradient
    wn = (w / w.sum()).reshape(-1)
    Om = ag.free_energy(E, p, wn, 0.1)
    ps = np.clip(p.cpu().numpy(), 1e-14, 1 - 1e-14)
    Sref = -np.sum(wn.cpu().numpy()[:, None].reshape(n, n, 1) * (ps * np.log(ps) + (1 - ps) * np.log1p(-ps)))
    assert abs(float(Om) - (ref - 0.1 * Sref)) < 1e-12 * max(1.0, abs(ref))

    def loss(P_, h_, S_, H_, p_):
        E_ = ag.hf_energy(P_, h=h_, Sigma=S_, H=H_, weights_b=wb, refP=refP)
        return ag.free_energy(E_, p_, wn, 0.1)

    xs = [t.detach().clone().requires_grad_(True) for t in (P, h, S, H, p)]
    grads = torch.autograd.grad(loss(*xs), xs)
    assert float(grads[4][0, 0, 0]) == 0.0
    for idx, name in enumerate(["P", "h", "Sigma", "H", "p"]):
        x0 = xs[idx].detach()
        d = _cplx(rng, x0.shape) if x0.is_complex() else _real(rng, x0.shape)
        if name == "p":
            d[0, 0, 0] = 0.0

        def f(x, idx=idx):
            args = [t.detach() for t in xs]
            args[idx] = x
            with torch.no_grad():
                return loss(*args)

        print(name, end=": ")
        _check_dir(f, x0, d, grads[idx])


def _density_exact_mu(F, w, n_e, T):
    """NumPy P(F) with mu solved to machine precision (brentq), occupations expit((mu - eps)/(T + 1e-12))."""
    from scipy.optimize import brentq
    from scipy.special import expit

    e, V = np.linalg.eigh(0.5 * (F + np.conj(np.swapaxes(F, -1, -2))))
    Tr = T + 1e-12
    cnt = lambda m: float(np.sum(w[..., None] * expit((m - e) / Tr))) - n_e
    mu = brentq(cnt, e.min() - 1.0, e.max() + 1.0, xtol=1e-16, rtol=1e-15, maxiter=500)
    f = expit((mu - e) / Tr)
    return (V * f[..., None, :]) @ np.conj(np.swapaxes(V, -1, -2)), mu


def test_density_from_fock_forward_and_backward(oracle):
    """Forward against NumPy eigh + the oracle's bisection; backward (electron count
    fixed) against central differences of the exact-mu map."""
    from cpp_hf_b200 import autograd as ag

    args, _P0, n_e = workloads.dirac(8, seed=2)
    rng = np.random.default_rng(7)
    F = torch.from_numpy(args["h"]).to(_dev()) + 0.05 * _cplx(rng, args["h"].shape, herm=True)
    w = torch.from_numpy(args["w2d"]).to(_dev())
    T = 0.1
    P, eps, mu = ag.density_from_fock(F, w, n_e, T)
    Fn = F.cpu().numpy()
    e, V = np.linalg.eigh(0.5 * (Fn + np.conj(np.swapaxes(Fn, -1, -2))))
    mu_ref = oracle.find_mu_bisection(e, args["w2d"], n_e, T)
    assert abs(float(mu) - mu_ref) < 1e-9
    f = 1.0 / (1.0 + np.exp((e - mu_ref) / (T + 1e-12)))
    Pref = (V * f[..., None, :]) @ np.conj(np.swapaxes(V, -1, -2))
    np.testing.assert_allclose(P.cpu().numpy(), Pref, atol=1e-9)
    C = _cplx(rng, F.shape)
    Fx = F.detach().clone().requires_grad_(True)
    L = (C.conj() * ag.density_from_fock(Fx, w, n_e, T)[0]).real.sum()
    (g,) = torch.autograd.grad(L, Fx)
    Cn = C.cpu().numpy()
    wn = args["w2d"]
    for trial in range(2):
        d = _cplx(rng, F.shape, herm=True).cpu().numpy()

        def loss(Fv):
            return float(np.sum(np.real(np.conj(Cn) * _density_exact_mu(Fv, wn, n_e, T)[0])))

        fd = (loss(Fn + H_FD * d) - loss(Fn - H_FD * d)) / (2 * H_FD)
        an = float(np.sum(np.real(np.conj(g.cpu().numpy()) * d)))
        print(f"density_from_fock: fd {fd:.12e} autograd {an:.12e}")
        assert abs(fd - an) <= 1e-6 * max(abs(fd), abs(an)) + 1e-10


def test_differentiation_workload_layered_96(native):
    """Backward of build_fock -> hf_energy -> free_energy w.r.t. P, H and V(q) on the
    layered model at 96x96, nb = 8, at a seeded random Hermitian P with eigenvalues in [0, 1]."""
    from cpp_hf_b200 import autograd as ag

    n = 96
    h_np, Vq_np, w_np = workloads.layered_model(n, n_layers=4, seed=0)
    P = torch.from_numpy(workloads.random_hermitian_density(n, 8, seed=1)).to(_dev())
    rng = np.random.default_rng(11)
    p = torch.from_numpy(rng.uniform(0.02, 0.98, size=(n, n, 8))).to(_dev())
    h = torch.from_numpy(h_np).to(_dev())
    Vq = torch.from_numpy(Vq_np).to(_dev())
    w = torch.from_numpy(w_np).to(_dev())
    wn = (w / w.sum()).reshape(-1)
    T = 0.05

    def loss(P_, h_, Vq_):
        VR = ag.vr_from_coulomb(Vq_, w)
        S_, H_, F_ = ag.build_fock(P_, h=h_, VR=VR, w2d=w, include_exchange=True)
        E_ = ag.hf_energy(P_, h=h_, Sigma=S_, H=H_, weights_b=w[..., None, None])
        return ag.free_energy(E_, p, wn, T)

    xs = [t.detach().clone().requires_grad_(True) for t in (P, h, Vq)]
    Om = loss(*xs)
    # value against the native build_fock_apply energy
    args = problem.kernel_args(w_np, h_np, Vq_np, T)
    _S, _H, _F, E_nat = native.build_fock_apply(args, P, None)
    ps = p.cpu().numpy()
    Sref = -np.sum(wn.cpu().numpy().reshape(n, n, 1) * (ps * np.log(ps) + (1 - ps) * np.log1p(-ps)))
    assert abs(float(Om) - (E_nat - T * Sref)) < 1e-10 * max(1.0, abs(E_nat))
    grads = torch.autograd.grad(Om, xs)
    for idx, name in enumerate(["P", "H", "V(q)"]):
        x0 = xs[idx].detach()
        d = _cplx(rng, x0.shape, herm=True) if x0.is_complex() else _real(rng, x0.shape)

        def f(x, idx=idx):
            a = [t.detach() for t in xs]
            a[idx] = x
            with torch.no_grad():
                return loss(*a)

        print(name, end=": ")
        _check_dir(f, x0, d, grads[idx])


def _layered_theta_model(n, seed=0):
    """theta = (U, Delta, gamma1) -> torch model dict; h affine in (Delta, gamma1), Vq linear in U."""
    h00, V1, w = workloads.layered_model(n, seed=seed, U=1.0, Delta=0.0, gamma1=0.0)
    hD, _, _ = workloads.layered_model(n, seed=seed, U=1.0, Delta=1.0, gamma1=0.0)
    hG, _, _ = workloads.layered_model(n, seed=seed, U=1.0, Delta=0.0, gamma1=1.0)
    dev = _dev()
    t_h0 = torch.from_numpy(h00).to(dev)
    t_hD = torch.from_numpy(hD - h00).to(dev)
    t_hG = torch.from_numpy(hG - h00).to(dev)
    t_V1 = torch.from_numpy(V1).to(dev)
    t_w = torch.from_numpy(w).to(dev)

    def model(theta):
        return {"h": t_h0 + theta[1] * t_hD + theta[2] * t_hG, "Vq": theta[0] * t_V1, "weights": t_w,
                "T": 0.05, "n_e": 4.0 * float(w.sum())}

    return model


# Central differences of the converged free energy re-solve at theta +- h,
# warm-started from the density converged at theta.  The SCF route (linear
# mixing) converges the layered model's residuals to 1e-12, so Omega* is exact
# far below the resolution of the 1e-5 step.


def _omega_fd(model, theta0, i, P0, method="scf"):
    from cpp_hf_b200 import autograd as ag

    vals = []
    for s in (+1, -1):
        th = theta0.clone()
        th[i] += s * H_FD
        info = ag.solve_model(model, th, method=method, P0=P0)
        assert info["converged"], info
        with torch.no_grad():
            vals.append(float(ag.free_energy_of(model, th.to(_dev()), info["P"], info["p"])))
    return (vals[0] - vals[1]) / (2 * H_FD)


@pytest.mark.parametrize("n", [24, 96])
def test_converged_free_energy_gradient_vs_finite_differences(native, n):
    """d Omega*/d(U, Delta, gamma1) at convergence vs central differences of GPU re-solves."""
    from cpp_hf_b200 import autograd as ag

    model = _layered_theta_model(n)
    theta0 = torch.tensor([1.0, 0.2, 0.4], dtype=torch.float64)
    Om, g, info = ag.free_energy_at_convergence(model, theta0)
    print(f"n={n}: {info['iterations']} SCF iterations, residual {info['residual']:.2e}")
    assert info["converged"]
    rels = []
    for i, name in enumerate(["U", "Delta", "gamma1"]):
        fd = _omega_fd(model, theta0, i, info["P"])
        rel = abs(fd - float(g[i])) / max(abs(fd), 1e-12)
        print(f"n={n} d Omega*/d {name}: autograd {float(g[i]):.10e} fd {fd:.10e} rel {rel:.2e}")
        rels.append(rel)
    assert max(rels) < 1e-6


def test_converged_free_energy_gradient_dm_route_matches_scf_route(native):
    """The direct-minimisation route reaches the same stationary point (12x12, where it converges)."""
    from cpp_hf_b200 import autograd as ag

    model = _layered_theta_model(12)
    theta0 = torch.tensor([1.0, 0.2, 0.4], dtype=torch.float64)
    Om_s, g_s, _ = ag.free_energy_at_convergence(model, theta0, method="scf")
    Om_d, g_d, info = ag.free_energy_at_convergence(model, theta0, method="dm")
    print(f"dm route: {info['iterations']} iterations, |dOmega| {abs(Om_s - Om_d):.2e}, "
          f"|dg| {float((g_s - g_d).abs().max()):.2e}")
    assert abs(Om_s - Om_d) < 1e-9 * max(1.0, abs(Om_s))
    assert float((g_s - g_d).abs().max()) < 1e-6 * float(g_s.abs().max())


def test_converged_free_energy_gradient_vs_oracle_resolves(oracle):
    """Same gradient against the oracle's solve_scf re-solved at theta +- h (12x12 mesh)."""
    from cpp_hf_b200 import autograd as ag

    n = 12
    model = _layered_theta_model(n)
    theta0 = torch.tensor([1.0, 0.2, 0.4], dtype=torch.float64)
    _Om, g, info = ag.free_energy_at_convergence(model, theta0)
    P_star = info["P"].cpu().numpy()
    rels = []
    for i, name in enumerate(["U", "Delta", "gamma1"]):
        vals = []
        for s in (+1, -1):
            th = theta0.clone()
            th[i] += s * H_FD
            m = model(th)
            w = m["weights"].cpu().numpy()
            args = problem.kernel_args(w, m["h"].cpu().numpy(), m["Vq"].cpu().numpy(), m["T"])
            out = oracle.solve_scf(args, P_star, m["n_e"], 2000, 1e-12, 1e-12, 0.5, 0.0, None, [], "linear", 6, 2,
                                   1.0, 0.0, False, True)
            assert out[5]
            # re-occupy the final Fock eigenbasis at the exact mu (brentq), as solve_model does
            P, _mu = _density_exact_mu(out[1], w, m["n_e"], m["T"] - 1e-12)
            p = np.linalg.eigvalsh(P)
            with torch.no_grad():
                vals.append(float(ag.free_energy_of(model, th.to(_dev()), torch.from_numpy(P).to(_dev()),
                                                    torch.from_numpy(p).to(_dev()))))
        fd = (vals[0] - vals[1]) / (2 * H_FD)
        rel = abs(fd - float(g[i])) / max(abs(fd), 1e-12)
        print(f"oracle d Omega*/d {name}: autograd {float(g[i]):.10e} fd {fd:.10e} rel {rel:.2e}")
        rels.append(rel)
    assert max(rels) < 1e-6
