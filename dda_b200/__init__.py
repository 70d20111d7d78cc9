"""dda_b200 -- discrete-dipole-approximation hot path on one NVIDIA B200.

The compute path is libdda_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/dda_cuda.h).  This package is the Python host side over that ABI;
it mirrors the reference's interfaces for the path:

  DDAParams            DDA/DDAParams.hpp:52-217 (grid, vector layout)
  CoupleConstants      DDA/DDAParams.hpp:222-242
  CudaMatVec           MatVec<T> / GpuMatVec<T> (DDA/MatVec.hpp:33-55,
                       DDA/GpuMatVec.hpp:42-100)
  CudaSolver           IterativeSolverBase<T>::getPolVec
                       (DDA/IterativeSolverBase.hpp:59) for qmr, bicgstab,
                       bicg and cgnr (DDA/DDAMain.cpp:647-656)

Beside them: postprocess (far field, Jones and Mueller matrices, cross
sections, Mie), cli (the DDA command line), matfile and datafiles (the
reference's MATLAB-style HDF5 and text data files, with no HDF5 library),
fielddiff and hdf5util (its FieldDiff and Hdf5Util tools), serve (the request
loop).

There is no CPU fallback: importing the package fails if the library cannot
be loaded, and every call raises DDAError with the library's message when the
device path fails (the reference throws Core::Exception the same way).
"""
from .api import (DDAError, Geometry, DDAParams, CoupleConstants, CudaMatVec, CudaSolver,
                  SOLVERS, PRECISIONS, fft_fit, beam_pol, beam_frame, Beam, lib, lib_path)

__all__ = ["DDAError", "Geometry", "DDAParams", "CoupleConstants", "CudaMatVec", "CudaSolver",
           "SOLVERS", "PRECISIONS", "fft_fit", "beam_pol", "beam_frame", "Beam", "lib",
           "lib_path"]
