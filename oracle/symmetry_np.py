"""NumPy restatement of cpp_hf's symmetry projector (src/cpp_hf/symmetry.py:18-117).

Test infrastructure: the checker the device projector (cpp_hf_b200.symmetry) is
compared against.  Parity pinned by the unchanged algorithm: group averages
(1/|G|) sum_g g A g^H over the unitary group, the same with A(-k) for the
spatial group (and the identity on A(k) when only a spatial group is given),
then the time-reversal average (A + U conj(A(-k)) U^H) / 2; -k is the "mod"
index (-i mod n) or the "flip" index (n - 1 - i) along the chosen axes.
"""

from __future__ import annotations

import numpy as np

__all__ = ["make_project_fn"]


def _minus_k(A, convention, axes):
    # symmetry.py:18-41
    if convention == "flip":
        return np.flip(A, axis=tuple(axes))
    if convention == "mod":
        n1, n2 = A.shape[0], A.shape[1]
        i = (-np.arange(n1)) % n1 if 0 in axes else np.arange(n1)
        j = (-np.arange(n2)) % n2 if 1 in axes else np.arange(n2)
        return A[i[:, None], j[None, :], ...]
    raise ValueError(f"k_convention must be 'mod' or 'flip', got {convention!r}")


def _conj_sum(A, G):
    # symmetry.py:44-50: sum_g g A g^H
    out = np.zeros_like(A)
    for g in G:
        out = out + (g @ A) @ np.conj(g.T)
    return out


def make_project_fn(*, unitary_group=None, spatial_group=None, spatial_k_convention="mod",
                    spatial_k_flip_axes=(0, 1), time_reversal_U=None, time_reversal_k_convention="mod",
                    time_reversal_k_flip_axes=(0, 1)):
    """symmetry.py:82-117."""
    if unitary_group is None and spatial_group is None and time_reversal_U is None:
        return lambda A: A
    G = None if unitary_group is None else np.asarray(unitary_group)
    S = None if spatial_group is None else np.asarray(spatial_group)
    U = None if time_reversal_U is None else np.asarray(time_reversal_U)

    def project(A):
        out = np.asarray(A)
        if G is not None or S is not None:
            same = G if G is not None else np.eye(S.shape[-1], dtype=S.dtype)[None]
            acc = _conj_sum(out, same)
            n = same.shape[0]
            if S is not None:
                acc = acc + _conj_sum(_minus_k(out, spatial_k_convention, spatial_k_flip_axes), S)
                n += S.shape[0]
            out = acc / n
        if U is not None:
            out = 0.5 * (out + U @ np.conj(_minus_k(out, time_reversal_k_convention, time_reversal_k_flip_axes))
                         @ np.conj(U.T))
        return out

    return project
