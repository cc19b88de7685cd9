"""GPU: the allocation-free chemical-potential entry point agrees with the workspace one.

``cpphf_find_mu_bisection_noalloc`` serves callers that cannot allocate device
memory when they call in (a fixed device-memory pool they may not grow, or a
latency-critical loop where cudaMalloc/cudaFree would synchronise the device).  Its scratch is a file-scope device array
shared by every call, so this test runs two different problems back to back
through the C ABI and compares each result with ``cpphf_find_mu_bisection``
(caller-provided workspace) at the tolerance the other mu tests use.  The file
name sorts last so a run stopping at the first failure has run everything else.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mu_with_workspace(lib, torch, bands, w, n_e, T):
    from cpp_hf_b200._native import _ptr, _stream, _ws

    nk, nb = bands.shape
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ws = _ws(lib.cpphf_mu_workspace_bytes(nk, nb))
    rc = lib.cpphf_find_mu_bisection(_ptr(bands), _ptr(w), nk, nb, n_e, T, 0, _ptr(out), _ptr(ws), ws.numel(),
                                     _stream())
    assert rc == 0, lib.cpphf_last_error()
    return float(out.item())


def _mu_noalloc(lib, torch, bands, w, n_e, T):
    from cpp_hf_b200._native import _ptr, _stream

    nk, nb = bands.shape
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.cpphf_find_mu_bisection_noalloc(_ptr(bands), _ptr(w), nk, nb, n_e, T, 0, _ptr(out), _stream())
    assert rc == 0, lib.cpphf_last_error()
    return float(out.item())


def test_noalloc_bisection_matches_workspace_entry_point_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cpp_hf_b200 import _lib

    lib = _lib.load()
    cases = [(36864, 8, 0.05, 3), (2304, 2, 0.1, 7)]  # two calls in a row, different sizes
    for nk, nb, T, seed in cases:
        rng = np.random.default_rng(seed)
        bands = torch.from_numpy(rng.normal(size=(nk, nb))).cuda()
        w = torch.full((nk,), 1.0 / nk, dtype=torch.float64, device="cuda")
        n_e = 0.5 * nb
        ref = _mu_with_workspace(lib, torch, bands, w, n_e, T)
        got = _mu_noalloc(lib, torch, bands, w, n_e, T)
        assert abs(got - ref) < 1e-12 * max(1.0, abs(ref)), (nk, nb, got, ref)


def test_noalloc_bisection_rejects_oversize_problems():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cpp_hf_b200 import _lib

    lib = _lib.load()
    rc = lib.cpphf_find_mu_bisection_noalloc(None, None, 1 << 28, 16, 1.0, 0.1, 0, None, None)
    assert rc == _lib.CPPHF_ERR_INVALID
    assert b"maximum" in lib.cpphf_last_error()
