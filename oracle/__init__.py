"""CPU oracle for the CBCT path (test infrastructure only).

``oracle.ctoracle`` wraps ``libctoracle.so`` (the C restatement in
``ct_oracle.c``) and ``_ref/libctref.so`` (the reference's own kernel sources
compiled for the CPU by ``ref_harness.cpp``).  Only the tests, the smoke
check and the benchmark's CPU-baseline leg import this package; the product
never does.
"""
