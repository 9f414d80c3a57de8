// micm/GPU.hpp -- micm's CUDA-path umbrella header (include/micm/GPU.hpp in
// micm), served by this library: with this include directory ahead of micm's,
// code written against micm's CUDA path (CudaSolverBuilderInPlace,
// CudaRosenbrockSolverParameters, CudaState, the system and process types)
// compiles against micm_b200 unchanged and links to libmicmb.so.
#pragma once

#include "../micm_b200/micm.hpp"
