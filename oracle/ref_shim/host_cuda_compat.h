// host_cuda_compat.h -- force-included when compiling the reference's CPU path
// with g++.  CPUlp.cuh pulls in method/hashtable.cuh and method/countmin.cuh
// (CUDA device code it never calls); these declarations only let them parse.
#pragma once
#include <climits>
#include <cstdint>
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
struct glp_shim_dim3 { unsigned x, y, z; };
static const glp_shim_dim3 threadIdx{0, 0, 0}, blockIdx{0, 0, 0}, blockDim{1, 1, 1}, gridDim{1, 1, 1};
template <class T, class U, class V> static inline T atomicCAS(T* a, U c, V v) { T o = *a; if (o == (T)c) *a = (T)v; return o; }
template <class T, class U> static inline T atomicAdd(T* a, U v) { T o = *a; *a = o + (T)v; return o; }
template <class T, class U> static inline T atomicDec(T* a, U v) { T o = *a; *a = (o == 0 || o > (T)v) ? (T)v : o - 1; return o; }
template <class T, class U> static inline T atomicExch(T* a, U v) { T o = *a; *a = (T)v; return o; }
template <class T> static inline T min(T a, T b) { return b < a ? b : a; }
