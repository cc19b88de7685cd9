#!/usr/bin/env python
"""Benchmark: Fock builds/s of the cpp_hf hot path on B200 (layered nb=8 model, 192x192 mesh).

One step = one Fock build (``build_fock_compact``: exchange FFT convolution +
assembly + energy) at a fixed seeded Hermitian density, FP64 (complex128).  The
layered model's V(q) is real and symmetric in the layer pair, so the build
takes the Hermitian-packed path (36 of the 64 orbital-pair channels, the
assembly and energy fused into the last FFT pass).  Inputs are device resident
for ``value``; ``e2e`` times the reference-facing drop-in call
``_native.build_fock_apply(kernel_args, P, None)`` with NumPy in and out (P
uploaded, Sigma, H and F downloaded every step; the kernel arrays' device
copies are reused between calls), and ``e2e_pipelined`` the repo's
``FockBuilder.build_host_async`` stream of builds (P in, F and E out, copies
overlapped with the builds).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

Multi-GPU (torchrun, one rank per GPU): independent replicas, no collective on
the data path ("scaling": "weak"); ``value`` is the builds of all ranks divided
by the slowest rank's device time.  ``--impl reference`` times the CPU oracle
(NumPy/SciPy FP64 restatement of the reference) on the host cores, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Fock builds/s & solves/s, nb=8 192^2 mesh, mixed vs FP64 GPU at dE<=1e-9"
UNIT = "Fock builds/s"
N_MESH = 192
N_LAYERS = 4
L2_FLUSH_BYTES = 256 << 20  # written between timed builds: twice the B200's 126 MB L2
WORKLOAD = "layered nb=8 (4 layers x A/B) model, 192x192 k-mesh, layer-resolved V(q) (192,192,8,8), FP64 Fock build"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--n", type=int, default=N_MESH)
    ap.add_argument("--solves", type=int, default=1, help="also time solve/solve_scf (1) or not (0)")
    ap.add_argument("--solve-reps", type=int, default=2)
    ap.add_argument("--oracle-solve", type=int, default=1, help="oracle DM solve estimate on the host")
    ap.add_argument("--sweep", type=int, default=96, help="batched-sweep instances (0 = skip)")
    ap.add_argument("--sweep-streams", type=int, default=16)
    ap.add_argument("--c64-mesh", type=int, default=144, help="nb=64 superlattice mesh (0 = skip)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    self.rows.append(parts)

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except ValueError:
                continue
            for nm, val in zip(names, r[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_uuid(torch, dev):
    try:
        u = torch.cuda.get_device_properties(dev).uuid
        s = str(u)
        return s if s.startswith("GPU-") else f"GPU-{s}"
    except Exception:
        return None


def cpu_baseline(args, P, n_builds):
    """Oracle build_fock_apply on the host cores (bounded sample)."""
    from oracle import native_np

    native_np.build_fock_apply(args, P, None)  # warm
    t0 = time.perf_counter()
    for _ in range(n_builds):
        native_np.build_fock_apply(args, P, None)
    dt = time.perf_counter() - t0
    return n_builds / dt, dt


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from cpp_hf_b200 import workloads

    args, _P0, _ne = workloads.layered(a.n, n_layers=N_LAYERS, seed=0)
    P = workloads.random_hermitian_density(a.n, 2 * N_LAYERS, seed=1)
    from oracle import native_np

    for _ in range(max(a.warmup, 0)):
        native_np.build_fock_apply(args, P, None)
    steps = max(1, min(a.steps, 100))
    t0 = time.perf_counter()
    for _ in range(steps):
        native_np.build_fock_apply(args, P, None)
    dt = time.perf_counter() - t0
    v = steps / dt
    cores = host_cores()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "nk": [a.n, a.n], "nb": 2 * N_LAYERS, "parallelism": "host threads"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{steps} oracle Fock builds (scipy.fft workers={cores}, numpy einsum)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _dm_call(native, args, P0, n_e, tol_E=1e-10, max_iter=1000):
    """cpp_hf's solve() defaults (SolverConfig, solver.py:19-64) with tol_E = 1e-10."""
    import torch

    nk1, nk2, nb = P0.shape[0], P0.shape[1], P0.shape[2]
    empty = torch.empty((0, nk1, nk2, nb, nb), dtype=torch.complex128, device=P0.device)
    return native.solve_dm(args, P0, n_e, max_iter, tol_E, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                           empty, 0.0, 1.0, [], None, False, True, False)


def _scf_call(native, args, P0, n_e, tol=1e-9, max_iter=1000):
    """solve_scf with linear mixing 0.5 and density/commutator tolerances `tol`."""
    return native.solve_scf(args, P0, n_e, max_iter, tol, tol, 0.5, 0.0, None, [], "linear", 6, 2, 1.0, 0.0,
                            True, False)


def time_solves(torch, native, args_dev, P0_dev, n_e, reps, n_mesh):
    """solves/s of solve (DM) and solve_scf at FP64 and switched precision, device resident."""
    stream = torch.cuda.current_stream()
    out = {}
    results = {}
    for kind, call in (("dm", _dm_call), ("scf", _scf_call)):
        for prec in ("fp64", "mixed"):
            a = dict(args_dev)
            if prec == "mixed":
                a["exchange_precision"] = "mixed"
            r = call(native, a, P0_dev, n_e)  # warm-up (and the result checked below)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                r = call(native, a, P0_dev, n_e)
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3 / reps
            E = r[5] if kind == "dm" else r[2]
            it = r[6] if kind == "dm" else r[4]
            conv = r[7] if kind == "dm" else r[5]
            results[(kind, prec)] = (E, r[2] if kind == "dm" else r[0])
            out[f"{kind}_{prec}"] = {"solves_per_s": 1.0 / t, "ms_per_solve": 1e3 * t, "iterations": int(it),
                                     "converged": bool(conv), "energy": float(E),
                                     "ms_per_iteration": 1e3 * t / max(int(it), 1)}
        e64, d64 = results[(kind, "fp64")]
        emx, dmx = results[(kind, "mixed")]
        out[f"{kind}_mixed"]["abs_dE_vs_fp64_gpu"] = abs(emx - e64)
        out[f"{kind}_mixed"]["speedup_vs_fp64"] = out[f"{kind}_mixed"]["solves_per_s"] / out[f"{kind}_fp64"]["solves_per_s"]
        g = oracle_goldens().get(kind) if n_mesh == N_MESH else None
        if g is not None:
            for prec in ("fp64", "mixed"):
                o = out[f"{kind}_{prec}"]
                o["oracle_energy"] = g["energy"]
                o["oracle_iterations"] = g["iterations"]
                o["abs_dE_vs_oracle"] = abs(o["energy"] - g["energy"])
                o["rel_dE_vs_oracle"] = abs(o["energy"] - g["energy"]) / abs(g["energy"])
    return out


def time_newton(torch, native, args_dev, P0_dev, n_e, reps=2, max_iter=60):
    """The trust-region Newton solve (optimizer=1, tol_grad=1e-6) of the same
    instance, FP64, device resident: time, outer iterations, final gradient norm."""
    nk1, nk2, nb = P0_dev.shape[0], P0_dev.shape[1], P0_dev.shape[2]
    empty = torch.empty((0, nk1, nk2, nb, nb), dtype=torch.complex128, device=P0_dev.device)

    def call():
        return native.solve_dm(args_dev, P0_dev, n_e, max_iter, 1e-7, 1e-6, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 1, 0.5,
                               20, empty, 0.0, 1.0, [], None, False, True, False)

    r = call()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        r = call()
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    it = int(r[6])
    return {"solves_per_s": 1.0 / t, "ms_per_solve": 1e3 * t, "iterations": it, "converged": bool(r[7]),
            "energy": float(r[5]), "final_grad_norm": float(r[9][-1]) if it else None,
            "ms_per_iteration": 1e3 * t / max(it, 1),
            "config": f"optimizer=newton, tol_grad=1e-6, max_iter={max_iter}, tr_delta0=0.5, tr_cg_max=20"}


def time_superlattice64(torch, native, dev, n):
    """The superlattice workload at nb = 64 (32 plane waves x 2 Dirac components,
    triangular superlattice, w0 = 0.1, scalar V with U = 0.5, T = 0.05, filling 32
    of 64) in its plain-mesh form (V(k - k') on every orbital pair, Hermitian
    channel packing: 2080 channels): one Fock build and one solve() (tol_E = 1e-10),
    device resident."""
    from cpp_hf_b200 import superlattice as sl
    from cpp_hf_b200.fock_builder import FockBuilder

    args, P0, n_e = sl.dirac_superlattice(n, n_pw=32, seed=0, streamed=False)
    fb = FockBuilder(args, precision=64)
    P = torch.zeros((n, n, 64, 64), dtype=torch.complex128, device=dev)
    P[..., :32, :32] = torch.eye(32, dtype=torch.complex128, device=dev)
    for _ in range(2):
        fb.build(P)
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(5):
        fb.build(P)
    e1.record(stream)
    torch.cuda.synchronize()
    t_build = e0.elapsed_time(e1) / 1e3 / 5
    del fb
    args_dev = {k: (torch.from_numpy(v).to(dev) if isinstance(v, np.ndarray) and v.size > 64 else v)
                for k, v in args.items()}
    P0_dev = torch.from_numpy(P0).to(dev)
    torch.cuda.synchronize()
    e0.record(stream)
    r = _dm_call(native, args_dev, P0_dev, n_e)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    return {"workload": f"Dirac superlattice, 32 plane waves x 2 (nb = 64), {n}x{n} mesh, plain-mesh form "
                        "(scalar V on every orbital pair, 2080 packed channels)",
            "ms_per_build": 1e3 * t_build, "solve_s": t, "iterations": int(r[6]), "converged": bool(r[7]),
            "energy": float(r[5]), "ms_per_iteration": 1e3 * t / max(int(r[6]), 1)}


def oracle_solve_estimate(args, P0_np, n_e, n_iter_gpu):
    """Oracle DM solve time from a bounded sample: init + 2 iterations, extrapolated to the
    iteration count of the FP64 GPU solve (the trajectories agree to ~1e-8)."""
    from oracle import native_np

    nk1, nk2, nb = P0_np.shape[0], P0_np.shape[1], P0_np.shape[2]
    empty = np.empty((0, nk1, nk2, nb, nb), np.complex128)

    def run(m):
        t0 = time.perf_counter()
        native_np.solve_dm(args, P0_np, n_e, m, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, empty, 0.0,
                           1.0, [], None, False, False, False)
        return time.perf_counter() - t0

    t1 = run(1)
    t3 = run(3)
    per_it = max((t3 - t1) / 2.0, 1e-9)
    base = max(t1 - per_it, 0.0)
    total = base + n_iter_gpu * per_it
    return 1.0 / total, per_it, base, t1 + t3


def load_traffic():
    """DRAM bytes per packed Fock build from the committed ncu summary of the 192x192 nb=8 build."""
    f = ROOT / "profiles" / "fock_packed_layered192_nb8.md"
    if not f.exists():
        return None
    m = re.search(r"^traffic_bytes_per_build:\s*(\d+)", f.read_text(), re.M)
    return {"nk": [N_MESH, N_MESH], "nb": 2 * N_LAYERS, "dram_bytes_per_build": int(m.group(1))} if m else None


def oracle_goldens():
    """Cached FP64 oracle solves of the 192x192 nb=8 workload (tests/golden, committed)."""
    out = {}
    for kind, name in (("dm", "dm_layered192.npz"), ("scf", "scf_layered192.npz")):
        f = ROOT / "tests" / "golden" / name
        if f.exists():
            g = np.load(f)
            out[kind] = {"energy": float(g["energy"]), "iterations": int(g["n_iter"])}
    return out


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    import torch

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}))
        return 1
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist

    from cpp_hf_b200 import _lib, _native, workloads
    from cpp_hf_b200.fock_builder import FockBuilder
    from cpp_hf_b200._native import _ptr, _stream, _ws

    lib = _lib.load()
    args, _P0, _ne = workloads.layered(a.n, n_layers=N_LAYERS, seed=rank)
    P_host_np = workloads.random_hermitian_density(a.n, 2 * N_LAYERS, seed=1 + rank)
    # exactly Hermitian blocks, C order (the sum with a transposed view is not)
    P_host_np = np.ascontiguousarray(0.5 * (P_host_np + np.conj(np.swapaxes(P_host_np, -1, -2))))
    fb = FockBuilder(args, precision=64, hermitian_density=True)
    if not fb.packed:
        raise RuntimeError("the layered workload should take the Hermitian-packed build")
    P = torch.from_numpy(P_host_np).to(dev)
    nk = a.n * a.n
    nb = 2 * N_LAYERS
    npk = nb * (nb + 1) // 2
    field = nk * nb * nb * 16
    stream = torch.cuda.current_stream()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    # L2 flush between timed builds: the packed build's inputs (101 MB) fit in the
    # 126 MB L2, so every timed build starts after a 256 MiB write
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def timed_flushed(fn, n):
        """Device time of n calls of fn (seconds, summed), the L2 flushed before each
        call and only the call itself between its pair of CUDA events."""
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        barrier()
        for e0, e1 in evs:
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
        barrier()
        return sum(e0.elapsed_time(e1) for e0, e1 in evs) / 1e3

    # ---- device-resident Fock builds as the solvers run them (Hermitian-packed,
    # assembly and energy fused, F and E out) ----
    for _ in range(max(3, a.warmup)):
        fb.build_fe(P)
    sampler = ClockSampler(gpu_uuid(torch, dev))
    barrier()
    sampler.start()
    for _ in range(max(3, a.warmup)):  # the sampler thread is up before the timed builds
        fb.build_fe(P)
    t_dev = timed_flushed(lambda: fb.build_fe(P), a.steps)
    # the public build_fock triple (exchange field written too), same flushing
    t_sigma = timed_flushed(lambda: fb.build(P), a.steps) / a.steps

    # ---- the full 64-channel path (any V, any P), for reference ----
    fb_full = FockBuilder(args, precision=64)
    VR = fb_full.dk._keep[1]
    Sig = torch.empty_like(P)
    xws = _ws(lib.cpphf_exchange_workspace_bytes(a.n, a.n, nb, 0, 64))

    def exch():
        _lib.check(lib.cpphf_exchange(_ptr(P), None, _ptr(VR), _ptr(Sig), a.n, a.n, nb, nb, 0, 0, 64,
                                      _ptr(xws), xws.numel(), _stream()), "exchange")

    def timed(fn, n):
        for _ in range(5):
            fn()
        return timed_flushed(fn, n) / n

    t_ex = timed(exch, a.steps)
    t_full_build = timed(lambda: fb_full.build(P), a.steps)
    del fb_full

    # ---- end to end through the drop-in call: NumPy in, NumPy out ----
    args_np = dict(args, hermitian_density=True)
    e2e_steps = max(3, min(a.steps, 30))
    e2e_E = []
    for _ in range(3):
        e2e_E.append(_native.build_fock_apply(args_np, P_host_np, None)[3])
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(e2e_steps):
        S_h, H_h, F_h, E_h = _native.build_fock_apply(args_np, P_host_np, None)
        e2e_E.append(E_h)
    g1.record(stream)
    barrier()
    t_e2e = g0.elapsed_time(g1) / 1e3

    # ---- end to end, pipelined stream of builds through FockBuilder ----
    P_pin = torch.from_numpy(P_host_np).pin_memory()
    F_pins = [torch.empty(fb.shape, dtype=torch.complex128).pin_memory() for _ in range(2)]
    E_pins = [torch.empty(1, dtype=torch.float64).pin_memory() for _ in range(2)]
    pipe_read = []

    def e2e_loop(n):
        fb.begin_host_pipeline()
        prev = None
        for i in range(n):
            ev = fb.build_host_async(P_pin, F_pins[i & 1], E_pins[i & 1])
            if prev is not None:
                prev[0].synchronize()  # the caller reads the previous step's result on the host
                pipe_read.append(float(E_pins[prev[1]][0]))
            prev = (ev, i & 1)
        fb.end_host_pipeline()
        prev[0].synchronize()
        pipe_read.append(float(E_pins[prev[1]][0]))

    e2e_loop(3)
    barrier()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    e2e_loop(e2e_steps)
    p1.record(stream)
    barrier()
    clocks = sampler.stop()
    t_pipe = p0.elapsed_time(p1) / 1e3

    # ---- solves/s (DM and SCF, FP64 and switched precision), device resident ----
    solves = None
    if a.solves:
        from cpp_hf_b200 import _native as native

        args_dev = {k: (torch.from_numpy(v).to(dev) if isinstance(v, np.ndarray) and v.size > 64 else v)
                    for k, v in args.items()}
        P0_dev = torch.from_numpy(np.ascontiguousarray(_P0)).to(dev)
        barrier()
        solves = time_solves(torch, native, args_dev, P0_dev, _ne, a.solve_reps, a.n)
        solves["newton_fp64"] = time_newton(torch, native, args_dev, P0_dev, _ne)
        if a.c64_mesh > 0:
            del args_dev, P0_dev
            torch.cuda.empty_cache()
            solves["superlattice_nb64"] = time_superlattice64(torch, native, dev, a.c64_mesh)
        barrier()

    # ---- batched sweep: concurrent streams (mixed and FP64) vs one by one in FP64 ----
    sweep = None
    if a.sweep > 0:
        from cpp_hf_b200 import batch

        inst = batch.upload(batch.sweep_instances(a.sweep, seed=rank))
        batch.solve_batch(inst[:4], precision="fp64", streams=1)  # warm-up (kernel attributes, allocator)
        barrier()
        seq, t_seq = batch.solve_batch(inst, precision="fp64", streams=1)
        bat64, t_bat64 = batch.solve_batch(inst, precision="fp64", streams=a.sweep_streams)
        bat, t_bat = batch.solve_batch(inst, precision="mixed", streams=a.sweep_streams)
        barrier()
        rel = [abs(x["energy"] - y["energy"]) / max(1.0, abs(x["energy"])) for x, y in zip(seq, bat)]
        same = [r for r in rel if r <= 1e-9]
        sweep = {
            "instances": len(inst),
            "batched_mixed_solves_per_s": len(inst) / t_bat,
            "batched_fp64_solves_per_s": len(inst) / t_bat64,
            "sequential_fp64_solves_per_s": len(inst) / t_seq,
            "speedup": t_seq / t_bat,
            "speedup_batched_fp64": t_seq / t_bat64,
            "mixed_same_state_as_fp64": len(same),
            "max_rel_dE_mixed_vs_fp64_same_state": max(same) if same else None,
            "max_rel_dE_mixed_vs_fp64_all": max(rel),
            "batched_fp64_matches_sequential": int(sum(abs(x["energy"] - y["energy"]) <= 1e-9 * max(1.0, abs(x["energy"]))
                                                        for x, y in zip(seq, bat64))),
            "converged_fp64": int(sum(bool(x["converged"]) for x in seq)),
            "converged_mixed": int(sum(bool(y["converged"]) for y in bat)),
            "iterations_fp64": int(sum(x["iterations"] for x in seq)),
            "iterations_mixed": int(sum(y["iterations"] for y in bat)),
            "streams": a.sweep_streams,
            "config": ("seeded instances: nb in {2,4,6,8} (Dirac for 2, layered for 4-8), mesh in "
                       "{36,48,72,96,144}^2, T~U[0.02,0.2], U~U[0.5,2], integer filling; solve() with tol_E=1e-10; "
                       "wall clock over the batch with device sync on both sides"),
        }

    # max over ranks
    times = torch.tensor([t_dev, t_ex, t_e2e, t_pipe, t_full_build], dtype=torch.float64, device=dev)
    if pg is not None:
        pg.all_reduce(times, op=pg.ReduceOp.MAX)
    t_dev, t_ex, t_e2e, t_pipe, t_full_build = [float(x) for x in times.cpu()]

    builds = a.steps * world
    value = builds / t_dev
    e2e = e2e_steps * world / t_e2e

    if rank == 0:
        peaks = {}
        pf = ROOT / "MEASURED_PEAKS.json"
        if pf.exists():
            peaks = json.loads(pf.read_text())
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        # algorithmic bytes of one packed build: the upper-triangle channels of P,
        # of the packed VR and of the packed Hermitian part of h are read, F written
        pk_bytes = (3 * npk + nb * nb) * 16 * nk
        ex_bytes = 3 * field  # full exchange: read P + read VR (dv = nb) + write Sigma
        fock_bytes_full = 5 * field  # full build: + read h + write F
        t_build = t_dev / a.steps
        achieved = pk_bytes / t_build / 1e9
        traffic = load_traffic()
        tr_val = None
        if traffic and traffic.get("nk") == [a.n, a.n] and traffic.get("nb") == nb:
            tr_val = traffic.get("dram_bytes_per_build")
        cb_v, cb_dt = None, None
        if world == 1 or rank == 0:
            import gc

            gc.collect()
            n_cpu = 10
            cb_v, cb_dt = cpu_baseline(args, P_host_np, n_cpu)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": a.steps,
            "warmup": a.warmup,
            "ms_per_step": 1e3 * t_build,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c128",
            "data": "synthetic (seeded layered model; P random Hermitian, eigenvalues in [0,1])",
            "config": {
                "workload": WORKLOAD, "nk": [a.n, a.n], "nb": nb, "exchange_channels": npk,
                "path": "Hermitian-packed build (V real symmetric, P Hermitian): 36 upper-triangle channels, "
                        "assembly and energy fused into the last FFT pass",
                "precision": "fp64", "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "l2": "L2 flushed before every timed build (256 MiB write outside the build's CUDA events); "
                      "the build's inputs and output (P, packed VR, packed h, F: 101 MB) fit in the 126 MB L2",
                "outputs": "F and E, as the solvers build (the exchange field is not written out)",
                "with_sigma": {"ms_per_build": 1e3 * t_sigma, "builds_per_s": 1.0 / t_sigma,
                               "note": "build_fock's public triple: the exchange field written too (+37.7 MB)"},
                "full_path": {"ms_per_build": 1e3 * t_full_build, "builds_per_s": 1.0 / t_full_build,
                              "exchange_ms": 1e3 * t_ex, "exchange_algorithmic_bytes": ex_bytes,
                              "exchange_frac": ex_bytes / t_ex / 1e9 / hbm,
                              "build_bytes": fock_bytes_full,
                              "note": "all 64 channels, separate assembly kernel (non-Hermitian V or P)"},
            },
            "roofline": {
                "kernel": "Hermitian-packed Fock build (3 launches: rows forward, columns * VR, rows inverse + "
                          "assembly + energy)",
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": tr_val, "algorithmic_bytes": pk_bytes,
                "peak_source": peak_src, "ms_per_launch": 1e3 * t_build,
            },
            "cpu_baseline": {"value": cb_v, "unit": UNIT, "cores": host_cores(), "kind": "port",
                             "sample": f"10 oracle Fock builds on the same 192^2 nb=8 instance "
                                       f"({cb_dt:.2f} s; scipy.fft workers = host cores)"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": field,
                    "d2h_bytes_per_step": 3 * field + 8,
                    "mode": "reference-facing _native.build_fock_apply: NumPy P in; NumPy Sigma, H, F and E out "
                            "(page-locked result buffers); kernel arrays' device copies reused between calls",
                    "host_energies_consistent": bool(len(set(e2e_E)) == 1 and all(map(math.isfinite, e2e_E)))},
            "e2e_pipelined": {"value": e2e_steps * world / t_pipe, "unit": UNIT, "h2d_bytes_per_step": field,
                              "d2h_bytes_per_step": field + 8,
                              "mode": "FockBuilder.build_host_async: copy-in, build and copy-out streams, two "
                                      "device buffer sets; the host reads every step's F and E",
                              "host_energies_consistent": bool(len(set(pipe_read)) == 1)},
            "gpu_launches": a.steps * fb.launches_per_build,
            "clocks": clocks,
        }
        if solves is not None:
            solves["config"] = ("solve(): SolverConfig defaults with tol_E=1e-10 (plateau window 5); "
                                "solve_scf(): linear mixing 0.5, density_tol=comm_tol=1e-9; "
                                "mixed = complex64 exchange until gradient norm / commutator residual < 1e-5, "
                                "then complex128; P0 and kernel arrays device resident; single solve per call")
            if a.oracle_solve and (world == 1 or rank == 0):
                v, per_it, base, spent = oracle_solve_estimate(args, _P0, _ne, solves["dm_fp64"]["iterations"])
                solves["cpu_baseline_dm"] = {
                    "solves_per_s": v, "cores": host_cores(), "kind": "port",
                    "sample": f"oracle solve_dm init + 1 and 3 iterations ({spent:.1f} s), extrapolated to "
                              f"{solves['dm_fp64']['iterations']} iterations: {per_it:.3f} s/iteration, "
                              f"{base:.3f} s setup"}
            line["solves"] = solves
        if sweep is not None:
            line["sweep"] = sweep
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
