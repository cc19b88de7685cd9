"""Batched sweeps: many independent Hartree-Fock solves of uneven mesh size and
band count run concurrently on one GPU.

The reference solves one problem per call on the host (``solver.solve``,
``reference_scf.solve_scf``).  Here a sweep (temperatures, fillings and
interaction strengths over Dirac and layered models) is packed onto the GPU:
every instance keeps its kernel arrays and solver workspace resident, and a
pool of host threads drives the instances on separate CUDA streams, largest
first, so that small meshes that cannot fill 148 SMs alone run side by side.
Each solve is the library's own device-resident solver (``_native.solve_dm`` /
``solve_scf``); the per-iteration convergence read-back only synchronises the
instance's own stream.  ``precision="mixed"`` runs each exchange in complex64
until the switch threshold and complex128 after it.
"""

from __future__ import annotations

import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native, workloads

__all__ = ["SweepInstance", "sweep_instances", "upload", "solve_batch"]


@dataclass
class SweepInstance:
    """One member of a sweep: model, mesh, band count, temperature, interaction, filling."""

    index: int
    model: str
    n: int
    nb: int
    T: float
    U: float
    filling: int
    args: dict
    P0: np.ndarray
    n_e: float
    dev: dict = field(default_factory=dict)

    @property
    def cost(self) -> float:
        return float(self.n * self.n * self.nb * self.nb)


def sweep_instances(count: int = 96, seed: int = 0, meshes=(36, 48, 72, 96, 144), bands=(2, 4, 6, 8)):
    """The seeded sweep: per instance, rng(seed + i) draws nb from `bands`, the mesh from
    `meshes`, T ~ U[0.02, 0.2], U ~ U[0.5, 2.0] and an integer filling in [1, nb - 1];
    nb = 2 is the Dirac model, nb = 4, 6, 8 the layered stack with nb / 2 layers."""
    out = []
    for i in range(count):
        r = np.random.default_rng(seed + i)
        nb = int(r.choice(bands))
        n = int(r.choice(meshes))
        T = float(r.uniform(0.02, 0.2))
        U = float(r.uniform(0.5, 2.0))
        filling = int(r.integers(1, nb))
        if nb == 2:
            args, P0, n_e = workloads.dirac(n, seed=seed + i, U=U, T=T)
            n_e = float(filling) * float(np.sum(args["w2d"]))
            model = "dirac"
        else:
            args, P0, n_e = workloads.layered(n, n_layers=nb // 2, seed=seed + i, U=U, T=T, filling=filling)
            model = "layered"
        out.append(SweepInstance(i, model, n, nb, T, U, filling, args, P0, n_e))
    return out


def upload(instances, device=None):
    """Copy every instance's kernel arrays and P0 to the device once (kept in inst.dev)."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    for inst in instances:
        d = {k: (torch.from_numpy(np.ascontiguousarray(v)).to(dev) if isinstance(v, np.ndarray) and v.size > 64
                 else v) for k, v in inst.args.items()}
        inst.dev = {"args": d, "P0": torch.from_numpy(np.ascontiguousarray(inst.P0)).to(dev)}
    torch.cuda.synchronize()
    return instances


def _solve_one(inst, precision, solver, tol, max_iter, graphs=True):
    args = dict(inst.dev["args"])
    if precision == "mixed":
        args["exchange_precision"] = "mixed"
    args["solve_graphs"] = graphs
    P0 = inst.dev["P0"]
    if solver == "dm":
        nb, n = inst.nb, inst.n
        empty = torch.empty((0, n, n, nb, nb), dtype=torch.complex128, device=P0.device)
        r = _native.solve_dm(args, P0, inst.n_e, max_iter, tol, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20,
                             empty, 0.0, 1.0, [], None, False, False, False)
        return {"energy": float(r[5]), "mu": float(r[4]), "iterations": int(r[6]), "converged": bool(r[7])}
    r = _native.solve_scf(args, P0, inst.n_e, max_iter, tol, tol, 0.5, 0.0, None, [], "linear", 6, 2, 1.0, 0.0,
                          False, False)
    return {"energy": float(r[2]), "mu": float(r[3]), "iterations": int(r[4]), "converged": bool(r[5])}


def solve_batch(instances, *, precision="mixed", solver="dm", streams=16, tol=1e-10, max_iter=1000):
    """Solve every instance; `streams` > 1 runs them concurrently on that many CUDA streams.

    Returns (results in instance order, wall seconds).  The wall clock brackets
    the whole batch with device synchronisation on both sides.
    """
    if not instances:
        return [], 0.0
    if not instances[0].dev:
        upload(instances)
    order = sorted(range(len(instances)), key=lambda i: -instances[i].cost)
    results = [None] * len(instances)
    dev = instances[0].dev["P0"].device
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    if streams <= 1:
        for i in order:
            results[i] = _solve_one(instances[i], precision, solver, tol, max_iter)
    else:
        # concurrent solves launch their kernels directly: per-solve graph
        # instantiation from many host threads contends in the driver
        local = threading.local()
        lock = threading.Lock()
        queue = list(order)

        def worker():
            if not hasattr(local, "stream"):
                torch.cuda.set_device(dev)
                local.stream = torch.cuda.Stream(device=dev)
            with torch.cuda.stream(local.stream):
                while True:
                    with lock:
                        if not queue:
                            break
                        i = queue.pop(0)
                    results[i] = _solve_one(instances[i], precision, solver, tol, max_iter, graphs=False)
            local.stream.synchronize()

        with ThreadPoolExecutor(max_workers=streams) as ex:
            futs = [ex.submit(worker) for _ in range(streams)]
            for f in futs:
                f.result()
    torch.cuda.synchronize(dev)
    return results, time.perf_counter() - t0
