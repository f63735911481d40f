"""ORACLE / TEST INFRASTRUCTURE ONLY.

Checkers for the tau00 path: ``reflib`` binds the reference's own C++
``calculateTauMatrix`` (compiled into ``oracle/_ref/libtauref.so`` by
``oracle/Makefile``) and ``port`` is a numpy restatement of the same algorithm.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference legs may import this package.  The product (``lsms_b200``) never does.
"""
