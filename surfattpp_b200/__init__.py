"""B200 engine for SurfATTPP's forward + adjoint misfit-gradient hot path.

Modules mirror the reference's call surfaces:
  eikonal   -- eikonal::FSM_UW_PS_lonlat_2d / FSM_O1_JSE_lonlat_2d / mask_uniform_grid
  preproc   -- preproc::forward_for_event (batched plan) and combine_kernels
  surfker   -- surfker::surfdisp / depthkernelHTI1d over many columns
  workloads -- seeded synthetic inputs
All numerical work runs in libsurfatt_gpu.so (sm_100a); there is no CPU path.
"""
__version__ = "0.1.0"
