"""B200 explicit residual engine for UCNS3D's SSP-RK3 stage.

Public pieces:

* ``ucns3d_b200.engine.Engine`` - the CUDA engine behind the C ABI of
  ``include/ucns3d_gpu.h`` (CALL_FLUX_SUBROUTINES_3D / RUNGE_KUTTA3 /
  CALCULATE_CFL of ``src/time_p.f90``).
* ``ucns3d_b200.mesh.Mesh`` - seeded synthetic meshes and their set-up tables
  (``include/ucns3d_prep.h``), for callers without UCNS3D's Fortran set-up.
* ``ucns3d_b200.config.make_config`` - ``ucg_config`` from UCNS3D.DAT-style
  parameters.
* ``ucns3d_b200.cases`` - the benchmark workloads.
"""
__all__ = ["engine", "mesh", "config", "cases", "build"]
