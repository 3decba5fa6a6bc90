"""ORACLE: FP64 CPU restatement of the Hotspice hot path, used only as a checker.

This package is test infrastructure. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference leg of ``bench.py`` may import it; the product package
``hotspice_b200`` never does, and it never stands in for the CUDA path.
"""
