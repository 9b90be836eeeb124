// Host stand-in for <device_launch_parameters.h> (checker build of the
// reference kernels only). The launcher in oracle/ref_launch.cpp walks the
// grid and sets these per OpenMP thread before calling a kernel body once
// per CUDA thread.
#pragma once
struct uint3 { unsigned int x, y, z; };
typedef uint3 dim3;
extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockDim;
extern thread_local uint3 gridDim;
