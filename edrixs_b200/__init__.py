"""edrixs_b200: a B200 (sm_100a) exact-diagonalisation core for the ED/XAS/RIXS path of EDRIXS.

Sub-modules
  io          file formats of the drop-in boundary (config.in, *.in, eigvec.N, poles, ...)
  fedrixs     drop-in ed_fsolver / xas_fsolver / rixs_fsolver / opavg_fsolver
  device      torch-facing wrappers of the CUDA kernels in libedx.so (include/edx.h)
  solvers     ground-state eigensolver (block thick-restart Lanczos) and Krylov drivers
  rixs        batched multi-shift RIXS (all incident energies, polarisations, ground states)
  serve       continuous-batching request loop with an HBM admission budget
  siam        seeded single-impurity Anderson model inputs for the workloads
"""
__version__ = "0.1.0"
