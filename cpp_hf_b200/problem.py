"""Kernel-argument precompute for the Fock-build path (host side, NumPy, once per problem).

Builds the ``kernel_args`` dict that cpp_hf's ``_native`` entry points consume
(keys of ``src/cpp_hf/solver.py:87-103``), restating the precompute of
``HartreeFockKernel.__init__`` (``src/cpp_hf/problem.py:24-228``):

* ``h`` as complex128, weights as float64, ``weight_sum = sum(w)``;
* an imaginary part of ``coulomb_q`` at or below 1e-8 is dropped
  (``problem.py:84-91``), and the Hermitian-channel-packing flag is set iff
  ``coulomb_q`` is ``(..., 1, 1)`` and real (``problem.py:92-94``);
* ``VR = FFT2(w * Vq) * exp(2*pi*i*(j*s0/n0 + l*s1/n1))`` with ``s = n // 2``
  so the exchange needs no ifftshift (``problem.py:95-104``);
* Hartree matrix, reference density and contact-term stacks
  (``problem.py:109-170``).

The embedded-reference-potential option (``problem.py:171-228``) is left to
the caller's own ``HartreeFockKernel``; this helper serves the synthetic
workloads and tests, which do not use it.
"""

from __future__ import annotations

import numpy as np


def shift_phase(n0: int, n1: int) -> np.ndarray:
    """``exp(2*pi*i*(j*s0/n0 + l*s1/n1))`` of ``problem.py:97-102``, shape (n0, n1)."""
    s0, s1 = n0 // 2, n1 // 2
    p0 = np.exp(2j * np.pi * np.arange(n0) * s0 / n0)
    p1 = np.exp(2j * np.pi * np.arange(n1) * s1 / n1)
    return p0[:, None] * p1[None, :]


def kernel_args(weights, hamiltonian, coulomb_q, T, *, include_hartree=False,
                include_exchange=True, reference_density=None, hartree_matrix=None,
                contact_terms=None) -> dict:
    """Return the ``kernel_args`` dict of ``solver._kernel_args_for_native``."""
    h = np.ascontiguousarray(np.asarray(hamiltonian), dtype=np.complex128)
    w2d = np.ascontiguousarray(np.asarray(weights), dtype=np.float64)
    n0, n1, nb = h.shape[0], h.shape[1], h.shape[-1]
    if not include_hartree and not include_exchange:
        raise ValueError("HartreeFockKernel must include at least one of Hartree or exchange.")
    if include_exchange:
        Vq = np.asarray(coulomb_q)
        if np.iscomplexobj(Vq):
            if float(np.max(np.abs(np.imag(Vq)))) <= 1e-8:
                Vq = np.real(Vq)
        else:
            Vq = Vq.astype(np.float64)
        hcp = bool(Vq.shape[-2:] == (1, 1) and not np.iscomplexobj(Vq))
        VR = np.fft.fftn(w2d[..., None, None] * Vq.astype(np.complex128, copy=False), axes=(0, 1))
        VR *= shift_phase(n0, n1)[..., None, None]
    else:
        hcp = False
        VR = np.zeros((n0, n1, 1, 1), dtype=np.complex128)
    if reference_density is not None:
        refP = np.ascontiguousarray(np.asarray(reference_density), dtype=np.complex128)
        if refP.shape != h.shape:
            raise ValueError(f"reference_density must have shape {h.shape}, got {refP.shape}")
        has_refP = True
    else:
        refP = np.empty((0,), dtype=np.complex128)
        has_refP = False
    if include_hartree:
        if hartree_matrix is None:
            raise ValueError("include_hartree=True requires hartree_matrix to be provided")
        if reference_density is None:
            raise ValueError("include_hartree=True requires reference_density to be provided")
        HH = np.asarray(hartree_matrix, dtype=np.float64)
        if HH.shape != h.shape[-2:]:
            raise ValueError(f"hartree_matrix must have shape {h.shape[-2:]}, got {HH.shape}")
    else:
        HH = np.zeros((nb, nb), dtype=np.float64)
    if not contact_terms:
        cg = np.zeros((1,), dtype=np.float64)
        cOi = np.zeros((1, nb, nb), dtype=np.complex128)
        cOj = np.zeros((1, nb, nb), dtype=np.complex128)
    else:
        cg = np.stack([np.asarray(t[0], dtype=np.float64) for t in contact_terms])
        cOi = np.stack([np.asarray(t[1], dtype=np.complex128) for t in contact_terms])
        cOj = np.stack([np.asarray(t[2], dtype=np.complex128) for t in contact_terms])
    return dict(
        h=h,
        VR=np.ascontiguousarray(VR, dtype=np.complex128),
        refP=refP,
        has_refP=has_refP,
        w2d=w2d,
        HH=np.ascontiguousarray(HH),
        contact_g=np.ascontiguousarray(cg),
        contact_Oi=np.ascontiguousarray(cOi),
        contact_Oj=np.ascontiguousarray(cOj),
        weight_sum=float(np.sum(w2d)),
        T=float(T),
        include_hartree=bool(include_hartree),
        include_exchange=bool(include_exchange),
        exchange_hcp=hcp,
    )
