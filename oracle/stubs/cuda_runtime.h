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
typedef struct CUstream_st* cudaStream_t;
#endif
