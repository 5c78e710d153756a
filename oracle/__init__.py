"""CPU oracle for the Cholesky path -- TEST INFRASTRUCTURE, never part of the product.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it.

  oracle.restated  -- ctypes wrapper of ddla_oracle.c, the plain-C restatement of
                      the reference's 1x1 CPU arm (LAPACK ?potf2 / BLAS ?trsm
                      algorithms, ppotrs ordering, DiagLogTerm reduction).
  oracle.lapack_arm -- the same arm through real LAPACK/BLAS (scipy's bundled
                      OpenBLAS): ?potrf_ then two ?trsm_, exactly the calls the
                      reference's CPU handle makes (src/Cholesky/potrf.cpp:46-49,
                      src/BLAS/trsm.cpp:139-140).  Used as the timed CPU baseline
                      and to cross-check the restatement at medium sizes.
"""
