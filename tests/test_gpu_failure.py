"""GPU: a bounded device wait that gives up reaches the caller as an error, and the
next call runs normally.

The grid barriers of the cooperative chemical-potential kernel poll a counter
at most ``cpphf_set_barrier_spin_limit`` times.  (Problems of up to 2^16
eigenvalues run as one thread-block cluster with hardware barriers instead, so
the cases below are larger.)  With a limit of one poll, the first blocks to
reach a barrier give up before the slower ones arrive (the problems below need
several hundred blocks), every block leaves the kernel
through the barrier's error flag, and the entry point reports
CPPHF_ERR_TIMEOUT (``RuntimeError`` in Python).  Nothing waits forever and no
copy is in flight in that kernel, so the context stays usable: the same call
with the default limit then returns the oracle's result.  (The mbarrier waits
on TMA copies are bounded too but are not driven to a timeout here: a copy
would still be in flight when the kernel returned.)
"""

from __future__ import annotations

import numpy as np
import pytest

from cpp_hf_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture
def tiny_barrier_limit():
    from cpp_hf_b200 import _lib

    lib = _lib.load()
    lib.cpphf_set_barrier_spin_limit(1)
    assert lib.cpphf_barrier_spin_limit() == 1
    try:
        yield lib
    finally:
        lib.cpphf_set_barrier_spin_limit(0)
        assert lib.cpphf_barrier_spin_limit() > 1


def test_find_mu_barrier_timeout_then_recovers(native, oracle, tiny_barrier_limit):
    rng = np.random.default_rng(11)
    nk, nb, T = 131072, 8, 0.05
    bands = rng.normal(size=(nk, nb))
    w = np.full(nk, 1.0 / nk)
    with pytest.raises(RuntimeError, match="gave up"):
        native.find_mu_bisection(bands, w, 0.5 * nb, T)
    tiny_barrier_limit.cpphf_set_barrier_spin_limit(0)
    mu = native.find_mu_bisection(bands, w, 0.5 * nb, T)
    ref = oracle.find_mu_bisection(bands, w, 0.5 * nb, T)
    assert abs(mu - ref) < 1e-12 * max(1.0, abs(ref))


def test_solve_dm_barrier_timeout_then_recovers(native, oracle, tiny_barrier_limit):
    # 576 x 576 Dirac mesh, nb = 2: 663 552 eigenvalues, a multi-block cooperative mu kernel
    args, P0, n_e = workloads.dirac(576, seed=0)
    defl = np.empty((0, 576, 576, 2, 2), np.complex128)
    call = (args, P0, n_e, 3, 1e-10, 0.0, 0.6, 0.5, 1e-3, 8, 10, 5, 25, 0, 0.5, 20, defl, 0.0, 1.0, [], None,
            False, False, False)
    with pytest.raises(RuntimeError, match="gave up|timeout"):
        native.solve_dm(*call)
    tiny_barrier_limit.cpphf_set_barrier_spin_limit(0)
    out = native.solve_dm(*call)
    ref = oracle.solve_dm(*call)
    assert out[6] == ref[6]
    assert abs(out[5] - ref[5]) < 1e-10 * max(1.0, abs(ref[5]))
