"""CPU oracle of the B200 backend.  TEST INFRASTRUCTURE ONLY.

Restates the reference (gbts/PyOP2) algorithms on the hot path, on the CPU:
the sequential backend's par_loop (:mod:`oracle.seq`), plan.pyx's partition,
staging and colouring (:mod:`oracle.plan`), build_sparsity_pattern_seq
(oracle_core.c) and, for pinning, the reference's own sparsity_utils.cxx
compiled unmodified (:mod:`oracle.reference`).  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it, as the
checker; the backend in pyop2_b200/ never imports it.
"""
