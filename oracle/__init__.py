"""CPU oracle for the cpp_hf Fock-build hot path (test infrastructure only).

Nothing in the product package imports this package; only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` do.
"""
