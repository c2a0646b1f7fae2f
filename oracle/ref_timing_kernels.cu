// ref_timing_kernels.cu -- TEST INFRASTRUCTURE ONLY: FlowLB's own solver
// kernels compiled for timing.
//
// src/cuda/lbmKernel2D.cu is compiled where it lies in the reference tree
// (included below, nothing copied), as FlowLB's own CMake build compiles it
// (separate compilation, nvcc's default floating-point contraction), except
// that its debug printf calls are compiled out: lbmKernel2D.cu:25 fires in
// FS_1 on every step and :83-117, :131, :146, :189, :210, :283, :302, :379-380,
// :407, :412 and :515 at fixed cells, which would time the device printf
// buffer instead of the solver.  Every printf statement there is a single
// call, so the macro below turns each into an empty expression statement.
// Linked with the same launch harness (ref_cuda_harness.cu) into
// oracle/_ref/libflbref_cuda_timing.so; the parity pin keeps the unmodified
// --fmad=false build (libflbref_cuda.so).
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <sys/types.h>

#include <cuda_runtime.h>

#include "cellCalculations.cuh"
#include "cudaInitData.cuh"
#include "lbmKernel2D.cuh"

#define printf(...) 0
#include "lbmKernel2D.cu"
#undef printf
