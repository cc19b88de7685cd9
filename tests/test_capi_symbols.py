"""CPU: the C-ABI library loads and exports every entry point ``include/*.h`` declares.

No compute call is made (this container has no GPU); the library is only
dlopen'ed and its symbols resolved.
"""

from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT
from cpp_hf_b200 import _lib

HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"typedef[^;]*\([^;]*;", "", text)  # function-pointer typedefs
        for m in re.finditer(r"\b(cpphf_[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["cpphf_exchange", "cpphf_build_fock", "cpphf_eigh_batched", "cpphf_find_mu_bisection",
                 "cpphf_solve_dm", "cpphf_solve_scf", "cpphf_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.fail(f"{_lib.LIB_PATH} not built (run python -m cpp_hf_b200.build)")
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_signatures_cover_header():
    declared = set(declared_functions())
    bound = set(_lib.exported_symbols())
    assert bound <= declared, bound - declared


def test_native_module_has_reference_names():
    from cpp_hf_b200 import _native
    from oracle import native_np

    assert sorted(_native.__all__) == sorted(native_np.__all__)
    import inspect

    for name in _native.__all__:
        a = inspect.signature(getattr(_native, name))
        b = inspect.signature(getattr(native_np, name))
        assert list(a.parameters) == list(b.parameters), name


def test_barrier_spin_limit_setting_round_trips():
    """Host-only setter (no device call): limit > 0 is kept, <= 0 restores the default."""
    if not _lib.LIB_PATH.exists():
        pytest.fail(f"{_lib.LIB_PATH} not built (run python -m cpp_hf_b200.build)")
    lib = _lib.load()
    default = lib.cpphf_barrier_spin_limit()
    assert default > 1000
    try:
        assert lib.cpphf_set_barrier_spin_limit(5) == 0
        assert lib.cpphf_barrier_spin_limit() == 5
    finally:
        lib.cpphf_set_barrier_spin_limit(0)
    assert lib.cpphf_barrier_spin_limit() == default
