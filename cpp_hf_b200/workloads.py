"""Seeded synthetic Hartree-Fock problems used by the parity tests and the benchmark.

No dataset is involved: the reference measures on no public suite, so the
benchmark workloads are fully specified synthetic models.

* ``dirac``: 2-band massive Dirac model on an n x n mesh over [-pi, pi)^2,
  ``H(k) = sin kx sx + sin ky sy + (m + 2 - cos kx - cos ky) sz`` plus a seeded
  Hermitian perturbation with N(0, noise^2) entries; scalar interaction
  ``V(q) = 2 pi U / (|q| + 0.05) * tanh(5 |q|)`` on the same centred grid.
* ``layered``: ``n_layers`` x {A, B} orbitals (index ``2 l + s``), intralayer
  ``f(k) = 1 + exp(i kx) + exp(i ky)`` between A_l and B_l, ``gamma1`` between
  A_{l+1} and B_l, a linear on-site ramp spanning ``Delta``, seeded
  N(0, noise^2) Hermitian noise; layer-resolved interaction
  ``V_{ll'}(q) = 2 pi U / (|q| + 0.05) * exp(-0.3 |q| |l - l'|)`` of shape
  (n, n, nb, nb).

Each builder returns ``(kernel_args, P0, n_electrons)`` ready for the
``_native`` entry points.
"""

from __future__ import annotations

import numpy as np

from .problem import kernel_args


def kgrid(n: int) -> np.ndarray:
    """k_i = -pi + 2 pi i / n."""
    return -np.pi + 2.0 * np.pi * np.arange(n) / n


def _herm_noise(rng, shape, sigma):
    A = rng.normal(0.0, sigma, size=shape) + 1j * rng.normal(0.0, sigma, size=shape)
    return 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))


def dirac(n: int = 48, *, seed: int = 0, m: float = -0.5, U: float = 1.0, T: float = 0.1,
          noise: float = 0.01):
    k = kgrid(n)
    kx, ky = np.meshgrid(k, k, indexing="ij")
    sx = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    sy = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    sz = np.array([[1, 0], [0, -1]], dtype=np.complex128)
    h = (np.sin(kx)[..., None, None] * sx + np.sin(ky)[..., None, None] * sy
         + (m + 2.0 - np.cos(kx) - np.cos(ky))[..., None, None] * sz)
    rng = np.random.default_rng(seed)
    h = h + _herm_noise(rng, h.shape, noise)
    q = np.sqrt(kx ** 2 + ky ** 2)
    Vq = (2.0 * np.pi * U / (q + 0.05) * np.tanh(5.0 * q))[..., None, None]
    w = np.full((n, n), 1.0 / (n * n))
    args = kernel_args(w, h, Vq, T, include_exchange=True, include_hartree=False)
    P0 = np.zeros_like(h)
    return args, P0, 1.0 * float(np.sum(w))


def layered_model(n: int = 192, *, n_layers: int = 4, seed: int = 0, U: float = 1.0, Delta: float = 0.2,
                  gamma1: float = 0.4, noise: float = 0.005):
    """(h, Vq, w) of the layered model; h is affine in (Delta, gamma1) and Vq linear in U."""
    nb = 2 * n_layers
    k = kgrid(n)
    kx, ky = np.meshgrid(k, k, indexing="ij")
    f = 1.0 + np.exp(1j * kx) + np.exp(1j * ky)
    h = np.zeros((n, n, nb, nb), dtype=np.complex128)
    for l in range(n_layers):
        a, b = 2 * l, 2 * l + 1
        h[..., a, b] = f
        h[..., b, a] = np.conj(f)
        ramp = Delta * ((l / (n_layers - 1) if n_layers > 1 else 0.0) - 0.5)
        h[..., a, a] += ramp
        h[..., b, b] += ramp
        if l + 1 < n_layers:
            a1 = 2 * (l + 1)
            h[..., a1, b] += gamma1
            h[..., b, a1] += gamma1
    rng = np.random.default_rng(seed)
    h = h + _herm_noise(rng, h.shape, noise)
    q = np.sqrt(kx ** 2 + ky ** 2)
    layer = np.arange(nb) // 2
    dl = np.abs(layer[:, None] - layer[None, :])
    Vq = 2.0 * np.pi * U / (q + 0.05)
    Vq = Vq[..., None, None] * np.exp(-0.3 * q[..., None, None] * dl[None, None])
    w = np.full((n, n), 1.0 / (n * n))
    return h, Vq, w


def layered(n: int = 192, *, n_layers: int = 4, seed: int = 0, U: float = 1.0, T: float = 0.05,
            Delta: float = 0.2, gamma1: float = 0.4, noise: float = 0.005, filling=None):
    h, Vq, w = layered_model(n, n_layers=n_layers, seed=seed, U=U, Delta=Delta, gamma1=gamma1, noise=noise)
    args = kernel_args(w, h, Vq, T, include_exchange=True, include_hartree=False)
    P0 = np.zeros_like(h)
    n_fill = n_layers if filling is None else int(filling)
    return args, P0, float(n_fill) * float(np.sum(w))


def random_hermitian_density(n: int, nb: int, *, seed: int = 0) -> np.ndarray:
    """Seeded Hermitian P(k) with eigenvalues in [0, 1] (the differentiation workload's P)."""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n, nb, nb)) + 1j * rng.normal(size=(n, n, nb, nb))
    Q, _ = np.linalg.qr(A)
    lam = rng.uniform(0.0, 1.0, size=(n, n, nb))
    return (Q * lam[..., None, :]) @ np.conj(np.swapaxes(Q, -1, -2))
