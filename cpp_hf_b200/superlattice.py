"""Superlattice (moire plane-wave) problems for the B200 library.

Host-side layout logic restated from cpp_hf ``superlattice.py`` (the extended
momentum grid of ``build_extended_layout``, superlattice.py:88-193, and the
superlattice_* kernel_args entries that ``SuperlatticeHartreeFockKernel`` hands
to the native solvers, superlattice.py:280-470 / solver.py:107-133), plus the
seeded 2-component Dirac superlattice used as the nb = 64 workload.

The Fock self-energy in the |k + G, alpha> basis,
    Sigma[a G_a, b G_b](k) = - sum_{q, G0} V(|k - q + G0|) rho[a (G_a + G0), b (G_b + G0)](q),
is a 2-D convolution in absolute momentum p = k - G on an extended fractional
grid that holds every tile k - G (zero padded to twice the support so the FFT
convolution is aperiodic), split into independent Delta-G = G_a - G_b channels.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .problem import kernel_args

__all__ = ["ExtendedLayout", "extended_layout", "superlattice_kernel_args", "dirac_superlattice"]


@dataclass(frozen=True)
class ExtendedLayout:
    """Index data of the extended grid (fields as in the reference's ExtendedGridLayout)."""

    N_ext_x: int
    N_ext_y: int
    n_supp_x: int
    n_supp_y: int
    g_a_off: np.ndarray         # (n_G, 2) int64 tile offsets in units of (nkx, nky)
    n_delta: int
    pair_to_delta: np.ndarray   # (n_G, n_G) int64
    V_lag_fft: np.ndarray       # (N_ext_x, N_ext_y) complex128, FFT of w * V on the lag grid
    delta_pair_count: np.ndarray
    delta_pair_i: np.ndarray
    delta_pair_j: np.ndarray
    delta_pair_start: np.ndarray


def extended_layout(g_frac, B, nkx, nky, coulomb_V, w_scalar) -> ExtendedLayout:
    """Extended-grid layout for a G basis ``g_frac`` (integer multiples of the
    reciprocal vectors, Cartesian G = B @ g) on an (nkx, nky) mesh
    (superlattice.py:88-193).

    The tile of plane wave G_a sits at offset -G_a (absolute momentum k - G_a);
    Delta-G channels are numbered in order of first appearance over (i, j)
    row-major and their (i, j) pairs listed in CSR form; the Coulomb kernel is
    tabulated on the FFT-natural lag grid of the extended cell (fractional lag
    / nk through B) and Fourier transformed with the weight ``w_scalar``.
    """
    g = np.asarray(g_frac, dtype=np.int64)
    n_G = g.shape[0]
    pos = -g
    lo = pos.min(axis=0)
    dim = pos.max(axis=0) - lo + 1
    n_supp_x, n_supp_y = int(nkx * dim[0]), int(nky * dim[1])
    N_ext_x, N_ext_y = 2 * n_supp_x, 2 * n_supp_y
    g_a_off = (pos - lo[None, :]).astype(np.int64)

    index = {}
    p2d = np.empty((n_G, n_G), dtype=np.int64)
    for i in range(n_G):
        for j in range(n_G):
            key = (int(g[i, 0] - g[j, 0]), int(g[i, 1] - g[j, 1]))
            p2d[i, j] = index.setdefault(key, len(index))
    n_delta = len(index)
    count = np.bincount(p2d.ravel(), minlength=n_delta).astype(np.int64)
    start = np.zeros(n_delta + 1, dtype=np.int64)
    start[1:] = np.cumsum(count)
    pi = np.empty(int(start[-1]), dtype=np.int64)
    pj = np.empty_like(pi)
    fill = start[:-1].copy()
    for i in range(n_G):
        for j in range(n_G):
            d = p2d[i, j]
            pi[fill[d]], pj[fill[d]] = i, j
            fill[d] += 1

    def lag(n_ext, nk):
        idx = np.arange(n_ext)
        return np.where(idx < n_ext // 2, idx, idx - n_ext).astype(float) / float(nk)

    fx, fy = np.meshgrid(lag(N_ext_x, nkx), lag(N_ext_y, nky), indexing="ij")
    B = np.asarray(B, dtype=float)
    qx = B[0, 0] * fx + B[0, 1] * fy
    qy = B[1, 0] * fx + B[1, 1] * fy
    V = np.asarray(coulomb_V(np.sqrt(qx ** 2 + qy ** 2)), dtype=float)
    V_fft = np.fft.fftn(float(w_scalar) * V, axes=(0, 1))
    return ExtendedLayout(N_ext_x, N_ext_y, n_supp_x, n_supp_y, g_a_off, n_delta, p2d,
                          np.ascontiguousarray(V_fft, dtype=np.complex128), count, pi, pj, start)


def superlattice_kernel_args(weights, hamiltonian, layout: ExtendedLayout, T, *, HH_GG=None, HH_GG_orbital=None,
                             V_lag_fft_orbital=None, include_hartree=True, include_exchange=True,
                             reference_density=None, hartree_degeneracy=1.0) -> dict:
    """kernel_args dict of a superlattice problem, as the reference's
    SuperlatticeHartreeFockKernel + _kernel_args_for_native build it: the mesh
    fields are placeholders (zero VR / HH / contact terms) and the
    superlattice_* entries carry the layout."""
    h = np.ascontiguousarray(np.asarray(hamiltonian), dtype=np.complex128)
    nkx, nky, D = h.shape[0], h.shape[1], h.shape[2]
    n_G = int(layout.g_a_off.shape[0])
    if D % n_G:
        raise ValueError(f"Hamiltonian dim D={D} not divisible by n_G={n_G} from layout")
    dim_orb = D // n_G
    w2d = np.ascontiguousarray(np.asarray(weights), dtype=np.float64)
    if HH_GG is None:
        HH_GG = np.zeros((n_G, n_G))
    args = kernel_args(w2d, h, np.zeros((nkx, nky, 1, 1)), T, include_hartree=False, include_exchange=True,
                       reference_density=reference_density)
    args.update(
        VR=np.zeros((nkx, nky, 1, 1), dtype=np.complex128),
        include_hartree=bool(include_hartree), include_exchange=bool(include_exchange), exchange_hcp=False,
        HH=np.zeros((D, D)),
        superlattice_fock_active=bool(include_exchange),
        superlattice_hartree_active=bool(include_hartree),
        hartree_degeneracy=float(hartree_degeneracy),
        n_G=n_G, dim_orb=int(dim_orb), n_delta=int(layout.n_delta),
        N_ext_x=int(layout.N_ext_x), N_ext_y=int(layout.N_ext_y),
        V_lag_fft=layout.V_lag_fft, g_a_off=layout.g_a_off,
        pair_i=layout.delta_pair_i, pair_j=layout.delta_pair_j, pair_start=layout.delta_pair_start,
        pair_to_delta=layout.pair_to_delta, HH_GG=np.ascontiguousarray(HH_GG, dtype=np.float64),
    )
    if HH_GG_orbital is not None:
        args["HH_GG_orbital"] = np.ascontiguousarray(HH_GG_orbital, dtype=np.float64)
    if V_lag_fft_orbital is not None:
        args["V_lag_fft_orbital"] = np.ascontiguousarray(V_lag_fft_orbital, dtype=np.complex128)
    return args


def _triangular_shells(n_pw):
    """The n_pw shortest vectors of the triangular lattice (integer coords), ordered by length then angle."""
    B = np.array([[1.0, 0.5], [0.0, np.sqrt(3.0) / 2.0]])
    r = int(np.ceil(np.sqrt(n_pw))) + 2
    cand = np.array([(a, b) for a in range(-r, r + 1) for b in range(-r, r + 1)], dtype=np.int64)
    cart = cand @ B.T
    L = np.round(np.hypot(cart[:, 0], cart[:, 1]), 9)
    ang = np.round(np.mod(np.arctan2(cart[:, 1], cart[:, 0]), 2 * np.pi), 9)
    order = np.lexsort((ang, L))
    return cand[order[:n_pw]], B


def dirac_superlattice(n=144, *, n_pw=32, seed=0, w0=0.1, U=0.5, T=0.05, streamed=True, hartree=False):
    """Seeded 2-component Dirac superlattice: n_pw plane waves k + G of a
    triangular superlattice (the shortest reciprocal vectors), diagonal blocks
    (k + G).sigma, a coupling w0 e^{i phi} (seeded phases) between G's that differ
    by a first-shell vector, scalar V(q) = 2 pi U / (|q| + 0.05) tanh(5 |q|),
    half filling (n_pw of 2 n_pw bands).

    Returns (kernel_args, P0, n_e) in the streamed superlattice form (the
    reference's SuperlatticeHartreeFockKernel; exchange only, or with
    ``hartree`` also the superlattice Hartree with HH_GG = V(|G_i - G_j|) and
    a zero diagonal) or, with
    ``streamed=False``, the plain-mesh form: the same h with V(k - k') over the
    mesh applied to every orbital pair (scalar V, Hermitian channel packing).
    """
    g, B = _triangular_shells(n_pw)
    rng = np.random.default_rng(seed)
    fk = np.arange(n) / n
    f1, f2 = np.meshgrid(fk, fk, indexing="ij")
    kx = B[0, 0] * f1 + B[0, 1] * f2
    ky = B[1, 0] * f1 + B[1, 1] * f2
    gc = g @ B.T
    D = 2 * n_pw
    h = np.zeros((n, n, D, D), dtype=np.complex128)
    for a in range(n_pw):
        px, py = kx + gc[a, 0], ky + gc[a, 1]
        h[..., 2 * a, 2 * a + 1] = px - 1j * py
        h[..., 2 * a + 1, 2 * a] = px + 1j * py
    first = 1.0
    for a in range(n_pw):
        for b in range(a + 1, n_pw):
            if abs(np.hypot(*(gc[a] - gc[b])) - first) < 1e-9:
                c = w0 * np.exp(1j * rng.uniform(0.0, 2.0 * np.pi))
                for s in range(2):
                    h[..., 2 * a + s, 2 * b + s] = c
                    h[..., 2 * b + s, 2 * a + s] = np.conj(c)
    w = np.full((n, n), 1.0 / (n * n))

    def coulomb(q):
        return 2.0 * np.pi * U / (q + 0.05) * np.tanh(5.0 * q)

    P0 = np.zeros_like(h)
    n_e = float(n_pw) * float(w.sum())
    if streamed:
        layout = extended_layout(g, B, n, n, coulomb, 1.0 / (n * n))
        HH = None
        if hartree:
            HH = coulomb(np.hypot(gc[:, None, 0] - gc[None, :, 0], gc[:, None, 1] - gc[None, :, 1]))
            np.fill_diagonal(HH, 0.0)
        args = superlattice_kernel_args(w, h, layout, T, HH_GG=HH, include_hartree=bool(hartree),
                                        include_exchange=True)
        return args, P0, n_e
    c = (np.arange(n) - n // 2) / n
    c1, c2 = np.meshgrid(c, c, indexing="ij")
    q = np.hypot(B[0, 0] * c1 + B[0, 1] * c2, B[1, 0] * c1 + B[1, 1] * c2)
    Vq = coulomb(q)[..., None, None]
    return kernel_args(w, h, Vq, T, include_exchange=True, include_hartree=False), P0, n_e
