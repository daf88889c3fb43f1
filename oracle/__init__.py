"""ORACLE -- test infrastructure only, never the product path.

CPU restatements of ac-fdtd's reference leapfrog (``leapfrog.py``, NumPy) and a ctypes driver
for the reference's own C backend compiled from its sources into ``oracle/_ref/`` (``ref_c.py``,
built by ``oracle/Makefile``). Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline and reference arms may import this package, and only as the checker or the timed
CPU baseline.
"""
