"""Symmetry projectors that run on the device (cpp_hf src/cpp_hf/symmetry.py:18-117).

``make_project_fn`` takes the reference's arguments and returns a
``DeviceProjector``: called on an array it averages over the unitary, spatial
and time-reversal symmetries with the library's CUDA kernels, and passed to a
solver as ``project_fn`` it is applied on the device inside the solve (no host
round trip per projection).  ``device_projector`` also recognises a projector
built by the reference's own ``cpp_hf.symmetry.make_project_fn`` (from the
arrays it closes over), so a reference user's symmetric solve takes the device
path unchanged; any other callable is left to the host callback.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check

__all__ = ["DeviceProjector", "make_project_fn", "device_projector"]

_CONVENTIONS = {"mod": 0, "flip": 1}


def _convention(name):
    name = str(name)
    if name not in _CONVENTIONS:
        raise ValueError(f"k_convention must be 'mod' or 'flip', got {name!r}")
    return _CONVENTIONS[name]


def _axes_mask(axes):
    axes = tuple(int(a) for a in axes)
    return (1 if 0 in axes else 0) | (2 if 1 in axes else 0)


class DeviceProjector:
    """Symmetry average of (nk1, nk2, nb, nb) fields on the current CUDA device."""

    def __init__(self, *, unitary_group=None, spatial_group=None, spatial_k_convention="mod",
                 spatial_k_flip_axes=(0, 1), time_reversal_U=None, time_reversal_k_convention="mod",
                 time_reversal_k_flip_axes=(0, 1)):
        self.s_conv = _convention(spatial_k_convention)
        self.t_conv = _convention(time_reversal_k_convention)
        self.s_axes = _axes_mask(spatial_k_flip_axes)
        self.t_axes = _axes_mask(time_reversal_k_flip_axes)
        dev = torch.device("cuda", torch.cuda.current_device())

        def up(x):
            if x is None:
                return None
            return torch.from_numpy(np.ascontiguousarray(np.asarray(x), dtype=np.complex128)).to(dev)

        self.G = up(unitary_group)
        self.S = up(spatial_group)
        self.U = up(time_reversal_U)
        if self.G is None and self.S is not None:
            # symmetry.py:106-108: a spatial group alone is averaged with the identity
            self.G = torch.eye(self.S.shape[-1], dtype=torch.complex128, device=dev)[None].contiguous()
        if self.G is not None and self.G.dim() == 2:
            self.G = self.G[None].contiguous()
        if self.S is not None and self.S.dim() == 2:
            self.S = self.S[None].contiguous()
        self._scratch = {}
        self._structs = {}

    @property
    def is_identity(self):
        return self.G is None and self.S is None and self.U is None

    def struct(self, nk1, nk2, nb):
        """The cpphf_symmetry record for fields of this shape (kept alive by self)."""
        key = (int(nk1), int(nk2), int(nb))
        if key not in self._structs:
            for M in (self.G, self.S):
                if M is not None and tuple(M.shape[-2:]) != (nb, nb):
                    raise ValueError(f"symmetry matrices are {tuple(M.shape[-2:])}, fields have nb = {nb}")
            if self.U is not None and tuple(self.U.shape) != (nb, nb):
                raise ValueError(f"time_reversal_U is {tuple(self.U.shape)}, fields have nb = {nb}")
            scratch = torch.empty(key + (nb,), dtype=torch.complex128, device=self._device())
            s = _lib.Symmetry()
            s.unitary_group = self.G.data_ptr() if self.G is not None else None
            s.n_unitary = 0 if self.G is None else int(self.G.shape[0])
            s.spatial_group = self.S.data_ptr() if self.S is not None else None
            s.n_spatial = 0 if self.S is None else int(self.S.shape[0])
            s.spatial_convention, s.spatial_axes = self.s_conv, self.s_axes
            s.time_reversal_U = self.U.data_ptr() if self.U is not None else None
            s.tr_convention, s.tr_axes = self.t_conv, self.t_axes
            s.scratch = scratch.data_ptr()
            self._scratch[key] = scratch
            self._structs[key] = s
        return self._structs[key]

    def _device(self):
        for M in (self.G, self.S, self.U):
            if M is not None:
                return M.device
        return torch.device("cuda", torch.cuda.current_device())

    def project_(self, A):
        """Project a contiguous complex128 CUDA tensor (nk1, nk2, nb, nb) in place."""
        if self.is_identity:
            return A
        nk1, nk2, nb = int(A.shape[0]), int(A.shape[1]), int(A.shape[2])
        s = self.struct(nk1, nk2, nb)
        lib = _lib.load()
        check(lib.cpphf_symmetry_project(C.byref(s), A.data_ptr(), nk1, nk2, nb,
                                         torch.cuda.current_stream().cuda_stream), "symmetry_project")
        return A

    def __call__(self, A):
        if isinstance(A, torch.Tensor) and A.is_cuda:
            return self.project_(A.to(torch.complex128).contiguous().clone())
        x = np.ascontiguousarray(np.asarray(A), dtype=np.complex128)
        t = torch.from_numpy(x).to(self._device())
        self.project_(t)
        torch.cuda.current_stream().synchronize()
        return t.cpu().numpy()


def make_project_fn(*, unitary_group=None, spatial_group=None, spatial_k_convention="mod",
                    spatial_k_flip_axes=(0, 1), time_reversal_U=None, time_reversal_k_convention="mod",
                    time_reversal_k_flip_axes=(0, 1)):
    """symmetry.py:82-117, on the device."""
    return DeviceProjector(unitary_group=unitary_group, spatial_group=spatial_group,
                           spatial_k_convention=spatial_k_convention, spatial_k_flip_axes=spatial_k_flip_axes,
                           time_reversal_U=time_reversal_U, time_reversal_k_convention=time_reversal_k_convention,
                           time_reversal_k_flip_axes=time_reversal_k_flip_axes)


# closure variables of the projector built by cpp_hf.symmetry.make_project_fn
_REF_CELLS = ("G", "S", "U", "s_k_conv", "s_k_axes", "t_k_conv", "t_k_axes")


def device_projector(fn):
    """The DeviceProjector equivalent of a project_fn, or None for a callable that
    is neither a DeviceProjector nor a projector of cpp_hf.symmetry.make_project_fn."""
    if isinstance(fn, DeviceProjector):
        return fn
    if getattr(fn, "__module__", None) != "cpp_hf.symmetry" or not callable(fn):
        return None
    code, cells = getattr(fn, "__code__", None), getattr(fn, "__closure__", None)
    if code is None:
        return None
    if fn.__qualname__.endswith("<lambda>") and not code.co_freevars:
        return DeviceProjector()  # make_project_fn without symmetries: the identity
    if not fn.__qualname__.startswith("make_project_fn.") or cells is None:
        return None
    vals = dict(zip(code.co_freevars, (c.cell_contents for c in cells)))
    if not all(name in vals for name in _REF_CELLS):
        return None
    return DeviceProjector(unitary_group=vals["G"], spatial_group=vals["S"], spatial_k_convention=vals["s_k_conv"],
                           spatial_k_flip_axes=vals["s_k_axes"], time_reversal_U=vals["U"],
                           time_reversal_k_convention=vals["t_k_conv"], time_reversal_k_flip_axes=vals["t_k_axes"])
