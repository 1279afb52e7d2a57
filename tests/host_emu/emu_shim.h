// Host stand-ins for the CUDA built-ins that the shared-memory FFT stages
// use, so that feram_b200/csrc/fft_smem.cuh compiles with a host compiler
// for the stage emulation in fft_stages_emu.cpp.  The emulation runs the
// threads of a stage one after another and the stages in order, so the
// barrier is empty.
#pragma once
#include <algorithm>
#include <cuda_runtime.h>

extern uint3 threadIdx, blockIdx;
extern dim3 blockDim, gridDim;
inline void __syncthreads() {}
inline unsigned long long __cvta_generic_to_shared(const void* p) { return (unsigned long long)p; }
template <class T>
inline T __ldg(const T* p) { return *p; }
inline int atomicCAS(int* a, int cmp, int v) {
  const int o = *a;
  if (o == cmp) *a = v;
  return o;
}
