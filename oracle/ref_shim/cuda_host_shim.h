// Host stand-ins for the CUDA runtime calls the reference makes, so that its sources
// (codec, operators, front end) build for the CPU with Thrust's host device systems
// (CPP or OMP): device memory becomes host memory. Test infrastructure only.
#pragma once
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <algorithm>
typedef int cudaError;
typedef int cudaError_t;
enum { cudaSuccess = 0 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
inline int cudaMalloc(void** p, size_t n) { *p = std::malloc(n ? n : 1); return 0; }
template <class T> inline int cudaMalloc(T** p, size_t n) { return cudaMalloc((void**)p, n); }
inline int cudaFree(void* p) { std::free(p); return 0; }
inline int cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { std::memmove(d, s, n); return 0; }
inline int cudaMemset(void* d, int v, size_t n) { std::memset(d, v, n); return 0; }
inline int cudaThreadSynchronize() { return 0; }
inline int cudaDeviceSynchronize() { return 0; }
inline const char* cudaGetErrorString(int) { return "shim"; }
inline int cudaHostAlloc(void** p, size_t n, unsigned) { *p = std::malloc(n ? n : 1); return 0; }
template <class T> inline int cudaHostAlloc(T** p, size_t n, unsigned f) { return cudaHostAlloc((void**)p, n, f); }
inline int cudaFreeHost(void* p) { std::free(p); return 0; }
inline int cudaMemGetInfo(size_t* f, size_t* t) { *f = *t = (size_t)180 << 30; return 0; }
#define cudaHostAllocDefault 0
inline long long __double2ll_rn(double x) { return (long long)std::llrint(x); }
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
struct int2 { int x, y; };
inline int2 make_int2(int x, int y) { return int2{x, y}; }
#include <thrust/functional.h>
#include <thrust/host_vector.h>
#include <thrust/device_vector.h>
#include <thrust/device_malloc.h>
#include <thrust/device_free.h>
#include <thrust/device_malloc_allocator.h>
