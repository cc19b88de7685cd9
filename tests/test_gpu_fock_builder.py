"""GPU: the device-resident FockBuilder (build, build_host and the pipelined
build_host_async) against the drop-in build_fock_apply and the oracle."""

from __future__ import annotations

import numpy as np
import pytest

from cpp_hf_b200 import workloads

pytestmark = pytest.mark.gpu


def test_fock_builder_host_paths_match_build_fock_apply(native, oracle):
    import torch

    from cpp_hf_b200.fock_builder import FockBuilder

    args, _P0, _ne = workloads.layered(24, seed=3)
    rng = np.random.default_rng(7)
    Ps = [workloads.random_hermitian_density(24, 8, seed=s) for s in (1, 2, 3, 4, 5)]
    fb = FockBuilder(args)
    ref = [native.build_fock_apply(args, P, None) for P in Ps]
    # synchronous host path
    F_pin = torch.empty(fb.shape, dtype=torch.complex128).pin_memory()
    E_pin = torch.empty(1, dtype=torch.float64).pin_memory()
    for P, r in zip(Ps, ref):
        fb.build_host(torch.from_numpy(P).pin_memory(), F_pin, E_pin)
        torch.cuda.current_stream().synchronize()
        np.testing.assert_array_equal(F_pin.numpy(), r[2])
        assert float(E_pin[0]) == float(r[3])
    # pipelined host path: one result buffer per step, every step checked
    P_pins = [torch.from_numpy(P).pin_memory() for P in Ps]
    F_out = [torch.empty(fb.shape, dtype=torch.complex128).pin_memory() for _ in Ps]
    E_out = [torch.empty(1, dtype=torch.float64).pin_memory() for _ in Ps]
    fb.begin_host_pipeline()
    events = [fb.build_host_async(P_pins[i], F_out[i], E_out[i]) for i in range(len(Ps))]
    fb.end_host_pipeline()
    events[-1].synchronize()
    for i, r in enumerate(ref):
        np.testing.assert_array_equal(F_out[i].numpy(), r[2])
        assert float(E_out[i][0]) == float(r[3])
    # and against the oracle
    o = oracle.build_fock_apply(args, Ps[0], None)
    np.testing.assert_allclose(F_out[0].numpy(), o[2], rtol=0, atol=1e-11 * np.max(np.abs(o[2])))
    assert abs(float(E_out[0][0]) - float(o[3])) < 1e-10 * max(1.0, abs(float(o[3])))
    del rng


def test_packed_builder_fe_matches_build_and_drop_in(native):
    """build_fe (F and E only, no exchange field written on the packed path) gives
    the same F and E as build() and as the drop-in call with hermitian_density."""
    import torch

    from cpp_hf_b200.fock_builder import FockBuilder

    args, _P0, _ne = workloads.layered(24, seed=4)
    P = workloads.random_hermitian_density(24, 8, seed=2)
    P = np.ascontiguousarray(0.5 * (P + np.conj(np.swapaxes(P, -1, -2))))
    fb = FockBuilder(args, hermitian_density=True)
    assert fb.packed
    Pd = torch.from_numpy(P).cuda()
    _S, F0, E0 = [x.clone() for x in fb.build(Pd)]
    F1, E1 = fb.build_fe(Pd)
    torch.cuda.synchronize()
    assert torch.equal(F0, F1) and float(E0) == float(E1)
    r = native.build_fock_apply(dict(args, hermitian_density=True), P, None)
    np.testing.assert_array_equal(F1.cpu().numpy(), r[2])
    assert float(E1) == float(r[3])
    with pytest.raises(ValueError):
        fb.build_fe(Pd.transpose(-1, -2))  # not C-contiguous
