"""Micro-benchmark / profiling driver for single hot-path operations.

    python -m cpp_hf_b200.kernel_bench --op exchange --n 192 --layers 4 --reps 5
    python -m cpp_hf_b200.kernel_bench --op build --n 192 --layers 4 --reps 5
    python -m cpp_hf_b200.kernel_bench --op build_packed --n 192 --layers 4 --reps 5

Runs ``--warmup`` untimed calls then ``--reps`` timed calls of one operation on
the seeded layered workload (device resident, current CUDA stream) and prints
the mean time per call from CUDA events.  Intended as the command under
``ncu`` (``-s`` = warm-up launches to skip).
"""

from __future__ import annotations

import argparse
import ctypes as C

import numpy as np
import torch

from . import _lib, workloads
from ._native import _DeviceKernel, _ptr, _stream, _ws


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", default="exchange",
                    choices=["exchange", "exchange32", "exchange_hcp", "build", "build_packed", "build_packed32", "eigh",
                             "mu", "solve_dm", "solve_scf", "solve_newton",
                             "sl_build", "sl_mesh_build", "sl_dm"])
    ap.add_argument("--pw", type=int, default=32, help="plane waves of the Dirac superlattice (sl_* ops)")
    ap.add_argument("--iters", type=int, default=10, help="solver iterations per call (solve_* ops)")
    ap.add_argument("--n", type=int, default=192)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if a.op.startswith("sl_"):
        return superlattice_op(a, lib, dev)
    nb = 2 * a.layers
    args, _P0, _ = workloads.layered(a.n, n_layers=a.layers, seed=0)
    P = torch.from_numpy(workloads.random_hermitian_density(a.n, nb, seed=1)).to(dev)
    dk = _DeviceKernel(args)
    VR = dk._keep[1]
    out = torch.empty_like(P)
    out2 = torch.empty_like(P)
    w = torch.empty((a.n, a.n, nb), dtype=torch.float64, device=dev)
    st = _stream()

    if a.op in ("exchange", "exchange32", "exchange_hcp"):
        prec = 32 if a.op == "exchange32" else 64
        hcp = 1 if a.op == "exchange_hcp" else 0
        V = VR if not hcp else VR[..., :1, :1].contiguous()
        dv = 1 if hcp else nb
        ws = _ws(lib.cpphf_exchange_workspace_bytes(a.n, a.n, nb, hcp, prec))

        def op():
            _lib.check(lib.cpphf_exchange(_ptr(P), None, _ptr(V), _ptr(out), a.n, a.n, nb, dv, hcp, 0, prec,
                                          _ptr(ws), ws.numel(), st), "exchange")
    elif a.op == "build":
        ws = _ws(lib.cpphf_build_fock_workspace_bytes(C.byref(dk.K)))
        E = torch.zeros(1, dtype=torch.float64, device=dev)

        def op():
            _lib.check(lib.cpphf_build_fock(C.byref(dk.K), _ptr(P), _ptr(out), _ptr(out2), None, _ptr(E), None,
                                            _ptr(ws), ws.numel(), st), "build")
    elif a.op in ("build_packed", "build_packed32"):
        # Hermitian-packed build as the solvers run it (no Sigma field written)
        if a.op == "build_packed32":
            dk.K.exchange_precision = 32
        if not dk.enable_packing():
            raise SystemExit("the packed build does not apply to this kernel")
        ws = _ws(lib.cpphf_build_fock_workspace_bytes(C.byref(dk.K)))
        E = torch.zeros(1, dtype=torch.float64, device=dev)

        def op():
            _lib.check(lib.cpphf_build_fock(C.byref(dk.K), _ptr(P), None, _ptr(out2), None, _ptr(E), None,
                                            _ptr(ws), ws.numel(), st), "build")
    elif a.op == "eigh":
        def op():
            _lib.check(lib.cpphf_eigh_batched(_ptr(P), _ptr(w), _ptr(out), a.n * a.n, nb, st), "eigh")
    elif a.op == "mu":
        bands = torch.randn((a.n * a.n, nb), dtype=torch.float64, device=dev)
        wt = torch.full((a.n * a.n,), 1.0 / (a.n * a.n), dtype=torch.float64, device=dev)
        mu = torch.zeros(1, dtype=torch.float64, device=dev)
        ws = _ws(lib.cpphf_mu_workspace_bytes(a.n * a.n, nb))

        def op():
            _lib.check(lib.cpphf_find_mu_bisection(_ptr(bands), _ptr(wt), a.n * a.n, nb, nb / 2.0, 0.05, 0,
                                                   _ptr(mu), _ptr(ws), ws.numel(), st), "mu")
    elif a.op in ("solve_dm", "solve_scf", "solve_newton"):
        from . import _native

        P0 = torch.zeros_like(P)

        def op():
            if a.op == "solve_newton":  # trust-region Newton, tol_grad 1e-6, at most --iters outer steps
                _native.solve_dm(args, P0, float(a.layers), a.iters, 1e-7, 1e-6, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 1,
                                 0.5, 20, None, 0.0, 1.0, [], None, True, True, True)
            elif a.op == "solve_dm":
                _native.solve_dm(args, P0, float(a.layers), a.iters, 0.0, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0,
                                 0.5, 20, None, 0.0, 1.0, [], None, True, True, True)
            else:
                _native.solve_scf(args, P0, float(a.layers), a.iters, 0.0, 0.0, 0.5, 0.0, None, [], "linear",
                                  6, 2, 1.0, 0.0, True, True)
    else:
        raise SystemExit(f"op {a.op} not wired")

    for _ in range(a.warmup):
        op()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        op()
    e1.record()
    torch.cuda.synchronize()
    print(f"{a.op} n={a.n} nb={nb}: {1e3 * e0.elapsed_time(e1) / a.reps:.2f} us/call")


def superlattice_op(a, lib, dev):
    """Fock builds / DM iterations of the 2-component Dirac superlattice (nb = 2 * pw):
    streamed superlattice form (sl_build, sl_dm) or plain-mesh form (sl_mesh_build)."""
    from . import _native, superlattice

    streamed = a.op != "sl_mesh_build"
    args, P0, n_e = superlattice.dirac_superlattice(a.n, n_pw=a.pw, seed=0, streamed=streamed)
    args = {k: (torch.from_numpy(v).to(dev) if isinstance(v, np.ndarray) and v.size > 4096 else v)
            for k, v in args.items()}
    nb = 2 * a.pw
    st = _stream()
    if a.op == "sl_dm":
        P0_t = torch.from_numpy(P0).to(dev)
        empty = torch.empty((0, a.n, a.n, nb, nb), dtype=torch.complex128, device=dev)

        def op():
            _native.solve_dm(args, P0_t, n_e, a.iters, 0.0, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty,
                             0.0, 1.0, [], None, False, False, False)
    else:
        dk = _DeviceKernel(args)
        rng = np.random.default_rng(1)
        lam = torch.from_numpy(rng.uniform(0.0, 1.0, size=(a.n, a.n, nb))).to(dev)
        P = torch.diag_embed(lam).to(torch.complex128)
        S = torch.empty_like(P)
        F = torch.empty_like(P)
        E = torch.zeros(1, dtype=torch.float64, device=dev)
        ws = _ws(lib.cpphf_build_fock_workspace_bytes(C.byref(dk.K)))

        def op():
            _lib.check(lib.cpphf_build_fock(C.byref(dk.K), _ptr(P), _ptr(S), _ptr(F), None, _ptr(E), None, _ptr(ws),
                                            ws.numel(), st), "build")
    for _ in range(a.warmup):
        op()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        op()
    e1.record()
    torch.cuda.synchronize()
    extra = f" iters={a.iters}" if a.op == "sl_dm" else ""
    print(f"{a.op} n={a.n} nb={nb}{extra}: {1e3 * e0.elapsed_time(e1) / a.reps:.2f} us/call")


if __name__ == "__main__":
    main()
