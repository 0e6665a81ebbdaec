"""cbmv_b200 -- CBMV's cost-volume path on NVIDIA B200 (sm_100a).

The reference (kbatsos/CBMV) drives three boost.python modules from its
Python drivers (test.py:30-35): libmatchers, libfeatextract and post, plus
scikit-learn's random forest.  This package offers drop-in modules with the
same names, functions and argument orders, backed by the CUDA kernels of
libcbmv.so (C ABI in include/cbmv.h):

    from cbmv_b200 import libmatchers as mtc, libfeatextract as fte, post
    from cbmv_b200.forest_gpu import GpuForest     # predict_proba drop-in
    from cbmv_b200.pipeline import StereoPipeline  # the fused test path

Inputs may be numpy arrays (host; results come back as numpy, like the
reference) or torch CUDA tensors (device-resident; results stay on the
device).
"""
__version__ = "0.1"
