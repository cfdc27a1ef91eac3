"""CPU oracle of the projector: TEST INFRASTRUCTURE ONLY.

A scalar C restatement of the reference projector's arithmetic
(``projector_oracle.c``) with a ctypes wrapper (``oracle.py``).  Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline arm of ``bench.py`` use it, always
as the checker or the timed CPU baseline, never inside the product path.
"""
