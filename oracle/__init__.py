"""ORACLE — test infrastructure, not the product.

CPU restatements of the reference's algorithms used only as the checker by
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py``. The ``glazier_b200`` package never imports this package.
"""
