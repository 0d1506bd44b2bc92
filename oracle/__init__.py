"""CPU oracle for the partially coherent imaging path (test infrastructure only).

Nothing in the product package imports this. Only ``tests/``, the smoke check in
``__graft_entry__.py`` and ``bench.py``'s CPU-baseline/reference arm use it, and
only as the checker or the timed CPU baseline.
"""
