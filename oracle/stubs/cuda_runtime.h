/* Host-only stand-in for <cuda_runtime.h>, used only by the oracle recipe
 * that compiles the reference's kernel sources as plain C++ so that their
 * bodies run on the CPU.  Each "launch" is emulated sequentially by the
 * harness, which sets the thread coordinates below before every call. */
#ifndef VFB_ORACLE_STUB_CUDA_RUNTIME_H
#define VFB_ORACLE_STUB_CUDA_RUNTIME_H
#define __host__
#define __device__
#define __global__
#define __shared__ static
#define __forceinline__ inline
struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;
inline void __syncthreads() {}
/* The global min / max overloads CUDA's math headers give host and device
 * code: same-type pairs, and a float paired with a double promoted to double. */
#include <cmath>
inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline double min(double a, double b) { return fmin(a, b); }
inline double max(double a, double b) { return fmax(a, b); }
inline double min(float a, double b) { return fmin((double)a, b); }
inline double max(float a, double b) { return fmax((double)a, b); }
inline double min(double a, float b) { return fmin(a, (double)b); }
inline double max(double a, float b) { return fmax(a, (double)b); }
/* and CUDA's float overload of log (the reference's wall model calls log on
 * a float in its single-precision build) */
inline float log(float x) { return logf(x); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
typedef struct CUstream_st* cudaStream_t;
#endif
