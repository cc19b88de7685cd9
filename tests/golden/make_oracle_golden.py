"""Write oracle outputs too slow to recompute inside the GPU tests.

``newton_layered192.npz``: the trust-region Newton solve (optimizer=1) of the
192x192, nb = 8 layered workload (seed 0, tol_grad 1e-6, max_iter 60) by
``oracle.native_np`` (about three minutes on one core): the energy and
gradient-norm histories, the final energy, the iteration count and the sum of
the occupations.

Usage: ``python tests/golden/make_oracle_golden.py``
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

import newton_cases as nc  # noqa: E402
from cpp_hf_b200 import workloads  # noqa: E402
from oracle import native_np  # noqa: E402

NEWTON_192 = dict(n=192, seed=0, tol_grad=1e-6, max_iter=60)


def newton_layered192():
    c = NEWTON_192
    args, P0, ne = workloads.layered(c["n"], seed=c["seed"])
    r = nc.solve(native_np, args, P0, ne, optimizer="newton", tol_grad=c["tol_grad"], max_iter=c["max_iter"])
    np.savez_compressed(HERE / "newton_layered192.npz", hist_E=r["hist_E"], hist_grad=r["hist_grad"],
                        energy=np.float64(r["energy"]), mu=np.float64(r["mu"]), n_iter=np.int64(r["n_iter"]),
                        converged=np.bool_(r["converged"]), p_sum=np.float64(np.sum(r["p"])))


if __name__ == "__main__":
    newton_layered192()
