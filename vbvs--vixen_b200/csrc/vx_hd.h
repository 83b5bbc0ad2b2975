// vx_hd.h - VX_HD marks helpers compiled for both the host and the device
// (plain inline functions in translation units that nvcc compiles as C++).
#pragma once

#ifdef __CUDACC__
#define VX_HD __host__ __device__ __forceinline__
#else
#define VX_HD inline
#endif

// Full unrolling of a fixed-trip loop in device code (keeps small per-thread
// arrays in registers); no effect on the host.
#ifdef __CUDA_ARCH__
#define VX_UNROLL _Pragma("unroll")
#else
#define VX_UNROLL
#endif
