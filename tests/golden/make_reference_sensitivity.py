"""Flag the recorded solver calls whose result the reference's own arithmetic
does not determine.

The reference's in-loop chemical-potential update (cpp_hf utils.hpp:79-116)
runs a fixed number of Newton steps inside a bracket.  Once Newton has
converged, the residual N(mu) - n_e is at the rounding level, and its sign
alone moves one end of the bracket to mu; the next Newton step then lands on
that end, the rule replaces it by the bracket's midpoint, and the remaining
steps bisect from there.  The mu that comes out, and with it the whole solver
trajectory (the iteration count and, when the run stops on the plateau test
during an oscillation, the final energy), can therefore change with the
summation order of N(mu).

This script re-runs every recorded ``solve_dm`` / ``solve_scf`` call of
``reference_calls.pkl.gz`` through the oracle with the chemical-potential
sums taken exactly (``math.fsum``) instead of NumPy's pairwise order, and
writes ``reference_calls_sensitive.json``: the calls whose iteration count or
energy changes, with both results and the amplitude of the runs' own energy
oscillation after their first two iterations (a run that stops on the plateau
test during an oscillation can stop anywhere within it).  The
GPU replay compares those calls at the spread the reference's arithmetic itself
leaves (see ``tests/test_gpu_reference_calls.py``).

    python tests/golden/make_reference_sensitivity.py
"""

from __future__ import annotations

import gzip
import json
import math
import pickle
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import native_np  # noqa: E402


def _expit(x):
    from scipy.special import expit

    return expit(x)


def mu_inloop_exact(eps, w_norm, n_target_norm, mu0, T, maxiter=25):
    """The oracle's _solve_mu_inloop with exactly rounded sums of N and Z."""
    eps = np.asarray(eps, dtype=np.float64)
    nb = eps.shape[-1]
    eps2 = eps.reshape(-1, nb)
    w = np.asarray(w_norm, dtype=np.float64).reshape(-1)[:, None]
    Tj = max(T, 1.0e-12)
    lo = float(eps2.min()) - 50.0 * Tj
    hi = float(eps2.max()) + 50.0 * Tj
    mu = min(max(mu0, lo), hi)
    for _ in range(int(maxiter)):
        p = _expit((mu - eps2) / Tj)
        N = math.fsum((w * p).ravel())
        Z = math.fsum((w * p * (1.0 - p) / Tj).ravel())
        g = N - n_target_norm
        if g < 0.0:
            lo = mu
        if g > 0.0:
            hi = mu
        mu_new = mu - g / max(Z, 1.0e-18)
        mu_bis = 0.5 * (lo + hi)
        if mu_new <= lo or mu_new >= hi:
            mu_new = mu_bis
        mu_new = min(max(mu_new, lo), hi)
        if not math.isfinite(mu_new):
            mu_new = mu_bis
        mu = mu_new
    return mu


def _summary(name, r):
    """(iterations, final energy, energy history) of a solver result tuple."""
    if name == "solve_dm":
        return int(r[6]), float(r[5]), np.asarray(r[8], dtype=np.float64)
    return int(r[4]), float(r[2]), np.asarray(r[6], dtype=np.float64)


def rerun_exact_full(call):
    """The call through the oracle with exact chemical-potential sums."""
    orig = native_np._solve_mu_inloop
    native_np._solve_mu_inloop = mu_inloop_exact
    try:
        r = getattr(native_np, call["name"])(*call["args"], **call["kwargs"])
    finally:
        native_np._solve_mu_inloop = orig
    return _summary(call["name"], r)


def rerun_exact(call):
    """(iterations, energy) of the call through the oracle with exact chemical-potential sums."""
    return rerun_exact_full(call)[:2]


def recorded(call):
    """(iterations, energy) the recorded run returned."""
    return _summary(call["name"], call["result"])[:2]


def late_amplitude(e_final, *histories):
    """The largest distance from the final energy that the runs' energies reach
    after their first two iterations (the initial descent): how far the
    reference's own trajectory oscillates on the input."""
    late = [h[2:] for h in histories if len(h) > 2]
    if not late:
        return 0.0
    return float(np.max(np.abs(np.concatenate(late) - e_final)))


def main() -> int:
    calls = pickle.load(gzip.open(HERE / "reference_calls.pkl.gz"))["calls"]
    out = {}
    for i, c in enumerate(calls):
        if c["name"] not in ("solve_dm", "solve_scf"):
            continue
        it0, e0, h0 = _summary(c["name"], c["result"])
        it1, e1, h1 = rerun_exact_full(c)
        if it1 != it0 or abs(e1 - e0) > 1e-12 * max(1.0, abs(e0)):
            amp = late_amplitude(e0, h0, h1)
            out[str(i)] = {"name": c["name"], "test": c["test"], "iterations": [it0, it1], "energy": [e0, e1],
                           "late_amplitude": amp}
            print(f"{i:3d} {c['name']} {c['test']}: iterations {it0} -> {it1}, energy {e0!r} -> {e1!r}, "
                  f"late oscillation {amp:.3e}", flush=True)
    (HERE / "reference_calls_sensitive.json").write_text(json.dumps(
        {"doc": "recorded solver calls whose oracle result changes when the chemical-potential sums are exact "
                "(make_reference_sensitivity.py)", "calls": out}, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
