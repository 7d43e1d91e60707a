"""CPU oracle for the EXAFS path-sum / PT-RMC hot path.

TEST INFRASTRUCTURE ONLY: this package is the checker. tests/, the smoke()
entry point and bench.py's cpu_baseline / --impl reference legs import it;
the chimera_b200 product never does.

  oracle.kernels   ctypes bindings to chx_oracle.c, the C restatement of the
                   reference's NVRTC kernels (exafs_gpu/kernels.py)
  oracle.host      NumPy restatements of the reference's host-side pieces:
                   the transform set-up (exafs_gpu/fourier.py), the profiled
                   chi^2 (methods/method_a_rmc.py), the supercell MS path
                   arrays (chimera/mslibrary.py)
  oracle.sampler   the plain PT-RMC loop (methods/method_a_rmc.py:250-455)
                   driving the C kernels: the CPU baseline
"""
