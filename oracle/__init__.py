"""Test infrastructure: the CPU oracle for the pptk hot path (see oracle.py).

Imported only by tests, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg; the product package never imports it."""
