// Host stand-in for <cuda_runtime.h>, used only when the reference's per-ray CUDA
// routine (src/cuda/rtKernels.cu) is compiled as plain host C++ into oracle/_ref.
// It supplies the launch built-ins as thread-local values that the host driver in
// oracle/ref_shim.cpp sets before calling the routine once per ray, and the
// device math wrappers that include/RT/precision.h only defines under nvcc.
#pragma once
#include <cmath>

#define __global__
#define __forceinline__ inline

struct ref_shim_dim3 {
    unsigned x, y, z;
};
extern thread_local ref_shim_dim3 blockIdx;
extern thread_local ref_shim_dim3 threadIdx;
extern thread_local ref_shim_dim3 blockDim;

inline float devAbs(float x) { return std::fabs(x); }
inline double devAbs(double x) { return std::fabs(x); }
inline float devFmax(float a, float b) { return std::fmax(a, b); }
inline double devFmax(double a, double b) { return std::fmax(a, b); }
inline float devFmin(float a, float b) { return std::fmin(a, b); }
inline double devFmin(double a, double b) { return std::fmin(a, b); }
