"""Oracle package -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this package, and only as a checker.  The product package
(hrnn_b200) never imports it.

* ``oracle.port``  : ctypes bindings of liboracle.so, the C restatement of the
                     reference's hot path (hrnn_oracle.c).
* ``oracle.ref``   : ctypes bindings of _ref/libhrnn_ref.so, the reference's own
                     include/hnswlib/hrnn.h compiled from its sources.
* ``oracle.idx``   : an independent numpy reader of the reference's .idx layout
                     (hrnn.h:861-1047).
* ``oracle.data``  : the seeded Gaussian-mixture generator and FP64 ground truth.
"""
