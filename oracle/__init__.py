"""CPU oracle for the GF2 Kadanoff-Baym hot path (test infrastructure only).

A C++ restatement of the reference solver (tblommel/NEdyson), used by tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg as the checker and
the timed CPU baseline.  The product library never imports, links or runs it.
"""
