// Build shim standing in for IMRTOpt/include/IMRTDoseMat.cuh when compiling
// IMRTgeom.cu: that file needs only the CUDA runtime and error-check helpers,
// not the Eigen/cuSPARSE matrix classes the real header pulls in.
#pragma once
#include "cuda_runtime.h"
#include "helper_cuda.h"
