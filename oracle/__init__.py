"""Test infrastructure only: the FP64 oracle and input generators used by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the checker.  Nothing in the
library (ascend-fft_b200/) imports, links or executes anything under oracle/.

Contents
  fft_oracle.py  numpy float64 (pocketfft) transforms with the reference's conventions,
                 the reference's acceptance metric and harness input modes, seeded generators
                 for the benchmark configurations.
  ref_fft.c      C restatement of the reference's FP64 oracle (src/framework/reference.cpp).
  kfft_fp32.c    C restatement of the fp32 arithmetic of the reference's AscendC kernels
                 (kfft_fwd, kfft_r2c_post, kfft_c2r_prep/post), standing in for the reference's
                 own fp32 output, which needs an Ascend NPU.
  Makefile       builds _build/liboracle.so from the restatements and, when the reference
                 sources are present, _ref/libref.so from the reference's own reference.cpp.
"""
