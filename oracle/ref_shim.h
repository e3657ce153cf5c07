// Host shim for compiling the reference's CUDA kernel sources as plain C++.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles
// Ops/FWI/Src_3d/{stress,velocity,stress_adj,velocity_adj,utilities}.cu from
// the reference tree, where they lie, with `g++ -x c++ -DUTILITIES_H__
// -include ref_shim.h`: defining the include guard skips the reference's
// utilities.h (which pulls CUDA, cuFFT and rapidjson headers) and this file
// supplies what the kernel bodies use instead.  __global__ functions become
// host functions; the launch geometry is read from thread-local variables
// that oracle/ref_driver.cpp sets before every emulated thread.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

#define REF_TLS __attribute__((tls_model("initial-exec"))) thread_local
extern REF_TLS dim3 blockIdx;
extern REF_TLS dim3 threadIdx;
extern REF_TLS dim3 blockDim;
extern REF_TLS dim3 gridDim;

#define __global__
#define __device__
#define __host__
#define __shared__ static
#define __constant__
inline void __syncthreads() {}

#define PI (3.141592653589793238462643383279502884197169)
