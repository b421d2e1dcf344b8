"""ORACLE — test infrastructure only.

The CPU restatement of NNPEngine's force step (``restate/nnpe_oracle.c``) and a harness around
the reference's own C++ compiled in place (``refshim/``, built into ``_ref/``). Only the tests,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this package, and only as
the checker; the product never loads it.
"""
