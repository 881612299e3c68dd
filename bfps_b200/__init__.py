"""bfps_b200: the NSVE / NSVEparticles hot path of bfps on B200 GPUs.

  solver    vorticity_equation, particles_system, NSVEparticles_step, ensemble
            (ctypes mirrors of the C-ABI in include/bfps_b200.h)
  dns       DNS: the launcher (bfps.DNS arguments, files and job loop)
  h5        HDF5 files without libhdf5
  serve     request loop over the batched engine
  ic        seeded synthetic initial conditions
  replicas  one-process-per-GPU helpers (independent instances)
  build     compiles csrc/bfps_b200.cu for sm_100a into _lib/libbfps_b200.so

Submodules are imported on use; importing the package loads no CUDA code.
"""
__version__ = "b200"
