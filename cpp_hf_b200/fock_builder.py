"""Device-resident Fock builder: repeated ``build_fock_compact`` calls without re-uploading the kernel.

``_native.build_fock_apply`` mirrors the reference and copies every kernel
array to the device on each call.  A loop that rebuilds the Fock matrix for
many densities on the same problem (an SCF / DM iteration, a benchmark) keeps
the kernel on the device instead:

    fb = FockBuilder(kernel_args)              # one upload
    Sigma, F, E = fb.build(P)                  # P: CUDA tensor (no copies) ...
    F, E = fb.build_fe(P)                      # ... F and E only, as the solvers build ...
    F_host, E = fb.build_host(P_pinned)        # ... or pinned host memory

A stream of builds from host memory (many densities, results read back each
time) pipelines the copies: ``begin_host_pipeline()``, then
``build_host_async(P_host, F_host, E_host)`` per density (it returns the event
after which F_host and E_host hold that result), then ``end_host_pipeline()``.  Two device buffer sets alternate; the upload of one
density runs while the previous result is downloaded (PCIe is full duplex) and
the build runs between them, each ordered by events.  A host buffer handed to
``build_host_async`` must stay untouched until ``end_host_pipeline()`` (or a
later synchronisation) returns.

Each ``build`` is one call of ``cpphf_build_fock`` on the current stream:
three exchange passes and the assembly kernel (which also reduces the energy),
or, on the Hermitian-packed path, three passes with the assembly and energy
fused into the last.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check
from ._native import _DeviceKernel, _ptr, _stream, _ws


class FockBuilder:
    """``hermitian_density=True`` declares that every density passed in is
    Hermitian: when V(q) is Hermitian too (real symmetric layer-resolved V,
    real scalar V) the build then transforms the nb(nb+1)/2 upper-triangle
    channels only, with the assembly fused into the last FFT pass
    (``packed`` tells whether that path is on)."""

    def __init__(self, kernel_args: dict, precision: int = 64, hermitian_density: bool = False):
        self.lib = _lib.load()
        self.dk = _DeviceKernel(kernel_args, precision=precision)
        self.dk.K.exchange_precision = int(precision)
        self.packed = bool(hermitian_density) and self.dk.enable_packing()
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
        pre = 2 if (K.include_hartree or K.has_contact) else 0
        if self.packed:
            return pre + 3  # rows forward, columns, rows inverse with the assembly and energy
        n = 1  # bulk assembly with the energy
        if K.include_exchange:
            n += 3
        return n + pre

    def _check_density(self, P: torch.Tensor):
        if not (isinstance(P, torch.Tensor) and P.is_cuda and P.dtype == torch.complex128
                and tuple(P.shape) == self.shape and P.is_contiguous()):
            raise ValueError(f"P must be a C-contiguous complex128 CUDA tensor of shape {self.shape}")

    def build(self, P: torch.Tensor):
        """Fock build at a device density P (complex128, C-contiguous, kernel shape)."""
        self._check_density(P)
        check(self.lib.cpphf_build_fock(C.byref(self.dk.K), _ptr(P), _ptr(self.Sigma), _ptr(self.F),
                                        _ptr(self.hd), _ptr(self.E), None, _ptr(self.ws), self.ws.numel(),
                                        _stream()), "build_fock")
        return self.Sigma, self.F, self.E

    def build_fe(self, P: torch.Tensor):
        """Fock build as the solvers run it: F and E only.  On the packed path the
        exchange field is then never written out (the full path still needs it as
        the assembly's input)."""
        self._check_density(P)
        self._build_into(P, self.F, self.E)
        return self.F, self.E

    def _build_into(self, P: torch.Tensor, F: torch.Tensor, E: torch.Tensor):
        sig = None if self.packed else _ptr(self.Sigma)
        check(self.lib.cpphf_build_fock(C.byref(self.dk.K), _ptr(P), sig, _ptr(F), _ptr(self.hd),
                                        _ptr(E), None, _ptr(self.ws), self.ws.numel(), _stream()), "build_fock")

    def begin_host_pipeline(self):
        """Start a pipelined sequence of host builds after the work already on the current stream."""
        if getattr(self, "_pipe", None) is None:
            dev = self.F.device
            self._pipe = {
                "s_in": torch.cuda.Stream(device=dev), "s_out": torch.cuda.Stream(device=dev),
                "P": [self.P_dev, torch.empty_like(self.P_dev)], "F": [self.F, torch.empty_like(self.F)],
                "E": [self.E, torch.zeros_like(self.E)],
            }
        pp = self._pipe
        pp["built"], pp["out"], pp["i"] = [None, None], [None, None], 0
        start = torch.cuda.Event()
        start.record(torch.cuda.current_stream())
        pp["s_in"].wait_event(start)

    def build_host_async(self, P_host: torch.Tensor, F_host: torch.Tensor, E_host: torch.Tensor):
        """One pipelined build: H2D of P on the copy-in stream, the build on the current
        stream, D2H of F and E on the copy-out stream (see the module docstring).
        Returns the CUDA event after which F_host and E_host hold the result."""
        pp = self._pipe
        if not (P_host.is_contiguous() and tuple(P_host.shape) == self.shape):
            raise ValueError(f"P_host must be a C-contiguous tensor of shape {self.shape}")
        b = pp["i"] & 1
        pp["i"] += 1
        cur = torch.cuda.current_stream()
        s_in, s_out = pp["s_in"], pp["s_out"]
        if pp["built"][b] is not None:
            s_in.wait_event(pp["built"][b])  # the build two steps back no longer reads P[b]
        with torch.cuda.stream(s_in):
            pp["P"][b].copy_(P_host, non_blocking=True)
        loaded = torch.cuda.Event()
        loaded.record(s_in)
        cur.wait_event(loaded)
        if pp["out"][b] is not None:
            cur.wait_event(pp["out"][b])  # F[b] and E[b] of two steps back are copied out
        self._build_into(pp["P"][b], pp["F"][b], pp["E"][b])
        built = torch.cuda.Event()
        built.record(cur)
        pp["built"][b] = built
        s_out.wait_event(built)
        with torch.cuda.stream(s_out):
            F_host.copy_(pp["F"][b], non_blocking=True)
            E_host.copy_(pp["E"][b], non_blocking=True)
        out = torch.cuda.Event()
        out.record(s_out)
        pp["out"][b] = out
        return out  # done once F_host and E_host hold this build's result

    def end_host_pipeline(self):
        """Order the current stream after every copy of the pipelined builds."""
        cur = torch.cuda.current_stream()
        for ev in self._pipe["out"]:
            if ev is not None:
                cur.wait_event(ev)

    def build_host(self, P_host: torch.Tensor, F_host: torch.Tensor, E_host: torch.Tensor):
        """End-to-end build from host memory: H2D of P, build, D2H of F and E (async on the stream)."""
        self.P_dev.copy_(P_host, non_blocking=True)
        self.build_fe(self.P_dev)
        F_host.copy_(self.F, non_blocking=True)
        E_host.copy_(self.E, non_blocking=True)
        return F_host, E_host
