"""B200-native (sm_100a) smoothed-profile-method step of KAPSEL.

Native code: kapsel3_b200/csrc (CUDA kernels + C ABI, include/kapsel_spm.h),
built in-tree into kapsel3_b200/_lib/libkapsel_spm.so.  Python modules:
  udf    -- UDF key files and seeded initial conditions
  spm    -- host mirror of the reference's solver interface (SPMRun)
  serve  -- continuous-batching request loop over many runs on one GPU
"""
