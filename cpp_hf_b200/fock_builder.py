"""Device-resident Fock builder: repeated ``build_fock_compact`` calls without re-uploading the kernel.

``_native.build_fock_apply`` mirrors the reference and copies every kernel
array to the device on each call.  A loop that rebuilds the Fock matrix for
many densities on the same problem (an SCF / DM iteration, a benchmark) keeps
the kernel on the device instead:

    fb = FockBuilder(kernel_args)              # one upload
    Sigma, F, E = fb.build(P)                  # P: CUDA tensor (no copies) ...
    F_host, E = fb.build_host(P_pinned)        # ... or pinned host memory

Each ``build`` is one call of ``cpphf_build_fock`` on the current stream
(three exchange passes, the assembly kernel and the energy sum).
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check
from ._native import _DeviceKernel, _ptr, _stream, _ws


class FockBuilder:
    def __init__(self, kernel_args: dict, precision: int = 64):
        self.lib = _lib.load()
        self.dk = _DeviceKernel(kernel_args, precision=precision)
        self.dk.K.exchange_precision = int(precision)
        nk1, nk2, nb = self.dk.shape
        self.shape = (nk1, nk2, nb, nb)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.Sigma = torch.empty(self.shape, dtype=torch.complex128, device=dev)
        self.F = torch.empty_like(self.Sigma)
        self.P_dev = torch.empty_like(self.Sigma)
        self.hd = torch.zeros(nb, dtype=torch.float64, device=dev)
        self.E = torch.zeros(1, dtype=torch.float64, device=dev)
        self.ws = _ws(self.lib.cpphf_build_fock_workspace_bytes(C.byref(self.dk.K)))

    @property
    def launches_per_build(self) -> int:
        K = self.dk.K
        n = 2  # assembly + energy sum
        if K.include_exchange:
            n += 3
        if K.include_hartree or K.has_contact:
            n += 2
        return n

    def build(self, P: torch.Tensor):
        """Fock build at a device density P (complex128, C-contiguous, kernel shape)."""
        check(self.lib.cpphf_build_fock(C.byref(self.dk.K), _ptr(P), _ptr(self.Sigma), _ptr(self.F),
                                        _ptr(self.hd), _ptr(self.E), None, _ptr(self.ws), self.ws.numel(),
                                        _stream()), "build_fock")
        return self.Sigma, self.F, self.E

    def build_host(self, P_host: torch.Tensor, F_host: torch.Tensor, E_host: torch.Tensor):
        """End-to-end build from host memory: H2D of P, build, D2H of F and E (async on the stream)."""
        self.P_dev.copy_(P_host, non_blocking=True)
        self.build(self.P_dev)
        F_host.copy_(self.F, non_blocking=True)
        E_host.copy_(self.E, non_blocking=True)
        return F_host, E_host
