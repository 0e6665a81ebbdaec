"""Oracle for the CBMV cost-volume path: TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg and
its reference arm) may import anything from here, and only as the checker or
as the timed CPU baseline.  The product (cbmv_b200) never calls into it.

  oracle.ref      ctypes bindings of the reference's own C++/CUDA sources,
                  compiled unmodified into oracle/_ref/ (see oracle/Makefile)
  oracle.cpu      ctypes bindings of oracle.c, a plain-C restatement of the
                  reference algorithms, with the same Python-facing names
  oracle.glue     Python-3 restatement of the reference's Python-2 drivers
                  (test.py / train.py) over either backend
"""
