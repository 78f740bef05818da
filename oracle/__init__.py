"""Test infrastructure: the CPU oracle for the polesitter FMM tick.

* ``oracle.oracle``  - ctypes binding of ``ps_oracle.c`` (the strict-IEEE
  restatement of the reference tick, with interaction-list introspection).
* ``oracle.refbind`` - ctypes binding of the reference itself compiled from
  its own header (``oracle/_ref``), used to pin the restatement.

Only ``tests/``, the smoke check and ``bench.py``'s CPU-baseline leg import
this package.
"""
