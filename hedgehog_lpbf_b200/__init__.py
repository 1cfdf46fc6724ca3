# SPDX-License-Identifier: 0BSD
"""hedgehog_lpbf_b200: B200-native 2D z-averaged explicit heat step for laser
powder bed fusion, a drop-in for hedgehog_lpbf's step kernels and GPU step
task.

Modules:
  params  -- Material/Process/Domain, StepConst/Partial/Tick ABI structs, make_const
  plan    -- laser plans (the reference single-track law and raster scans)
  build   -- nvcc build of liblpbf_b200.so (sm_100a)
  _lib    -- ctypes binding of the C-ABI
  solver  -- device-resident field advancing along a plan (torch for memory)
"""
__version__ = "0.1.0"
