// enstrophy.cu -- the enstrophy analyzer's node values and their FP64 sum.
//
// EnstrophyAnalyzer::run (src/gpu/core/PostProcessor/EnstrophyAnalyzer.cu:63-98)
// computes the macroscopic fields, then per fluid node 1/2 (drho + 1) |curl u|^2
// (:112-338) and reports the sum over the nodes that had all six axis
// neighbours fluid, divided by their number.  The node value follows the
// reference's arithmetic in the working precision; the sum is FP64 (the
// reference reduces in the working precision with thrust, in an unspecified
// order).  The reduction is a grid-stride loop with one FP64 partial pair per
// block, like the mass / energy sums.
#include <cuda_runtime.h>

#include <vector>

#include "capi_common.cuh"
#include "d3q27.cuh"

namespace vfb
{
namespace
{
constexpr uint32_t kFluid = 19u;
constexpr int kEnstrophyThreads = 256;

struct AxisWalk {
    const uint32_t* nX;
    const uint32_t* nY;
    const uint32_t* nZ;
    const uint32_t* nNeg;
    __host__ __device__ uint32_t plus(int axis, uint32_t k) const
    {
        return axis == 0 ? nX[k] : axis == 1 ? nY[k] : nZ[k];
    }
    // the negative neighbour: the -x-y-z neighbour, then two positive steps
    __host__ __device__ uint32_t minus(int axis, uint32_t k) const
    {
        const uint32_t w = nNeg[k];
        return axis == 0 ? nZ[nY[w]] : axis == 1 ? nZ[nX[w]] : nY[nX[w]];
    }
};

// central difference of the given order (EnstrophyAnalyzer.cu:285-327), with
// the reference's constant products and operation order
template <class R>
__host__ __device__ inline R centralDifference(const R* u, const uint32_t* P, const uint32_t* M, int order)
{
    if (order == 2)
        return (u[P[0]] - u[M[0]]) / R(2);
    if (order == 4)
        return ((R(8) * u[P[0]] - R(8) * u[M[0]]) - (u[P[1]] - u[M[1]])) / R(12);
    if (order == 6)
        return ((R(5) * R(9)) * (u[P[0]] - u[M[0]]) - R(9) * (u[P[1]] - u[M[1]]) + (u[P[2]] - u[M[2]])) /
               (R(6) * R(10));
    return ((R(28) * R(8)) * (u[P[0]] - u[M[0]]) - (R(7) * R(8)) * (u[P[1]] - u[M[1]]) +
            (R(8) * R(4) * (R(1) / R(3))) * (u[P[2]] - u[M[2]]) - (u[P[3]] - u[M[3]])) /
           (R(7) * R(10) * R(4));
}

// one node: false when it is not counted (not fluid, or an axis neighbour is
// not fluid); each axis takes the widest stencil (8, 6, 4, 2) on fluid nodes
template <class R>
__host__ __device__ inline bool enstrophyAtNode(const R* rho, const R* vx, const R* vy, const R* vz,
                                                const uint32_t* geo, const AxisWalk& walk, uint32_t k, R& value)
{
    if (geo[k] != kFluid)
        return false;
    uint32_t P[3][4], M[3][4];
    int order[3] = { 8, 8, 8 };
    bool reach = true;
    for (int a = 0; a < 3; ++a) {
        P[a][0] = walk.plus(a, k);
        M[a][0] = walk.minus(a, k);
        reach = reach && geo[P[a][0]] == kFluid && geo[M[a][0]] == kFluid;
    }
    if (!reach)
        return false;
    for (int a = 0; a < 3; ++a) {
        for (int i = 1; i < 4; ++i) {
            P[a][i] = walk.plus(a, P[a][i - 1]);
            M[a][i] = walk.minus(a, M[a][i - 1]);
            if ((geo[P[a][i]] != kFluid || geo[M[a][i]] != kFluid) && order[a] > 2 * i)
                order[a] = 2 * i;
        }
    }
    const R dxvy = centralDifference(vy, P[0], M[0], order[0]);
    const R dxvz = centralDifference(vz, P[0], M[0], order[0]);
    const R dyvx = centralDifference(vx, P[1], M[1], order[1]);
    const R dyvz = centralDifference(vz, P[1], M[1], order[1]);
    const R dzvx = centralDifference(vx, P[2], M[2], order[2]);
    const R dzvy = centralDifference(vy, P[2], M[2], order[2]);
    const R wx = dyvz - dzvy, wy = dzvx - dxvz, wz = dxvy - dyvx;
    value = R(0.5) * (rho[k] + R(1)) * (wx * wx + wy * wy + wz * wz);
    return true;
}

template <class R>
__global__ void __launch_bounds__(kEnstrophyThreads)
    enstrophyKernel(const R* __restrict__ rho, const R* __restrict__ vx, const R* __restrict__ vy,
                    const R* __restrict__ vz, unsigned long long N, const uint32_t* __restrict__ geo, AxisWalk walk,
                    double* __restrict__ partial)
{
    double sum = 0.0, count = 0.0;
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < N;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        R v;
        if (enstrophyAtNode<R>(rho, vx, vy, vz, geo, walk, (uint32_t)k, v)) {
            sum += (double)v;
            count += 1.0;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        count += __shfl_down_sync(0xffffffffu, count, o);
    }
    __shared__ double sm[2][kEnstrophyThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sm[0][warp] = sum;
        sm[1][warp] = count;
    }
    __syncthreads();
    if (warp == 0) {
        sum = lane < kEnstrophyThreads / 32 ? sm[0][lane] : 0.0;
        count = lane < kEnstrophyThreads / 32 ? sm[1][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sum += __shfl_down_sync(0xffffffffu, sum, o);
            count += __shfl_down_sync(0xffffffffu, count, o);
        }
        if (lane == 0) {
            partial[2 * blockIdx.x + 0] = sum;
            partial[2 * blockIdx.x + 1] = count;
        }
    }
}

template <class R>
void nodesOnHost(const void* rho, const void* vx, const void* vy, const void* vz, unsigned long long N,
                 const uint32_t* geo, const AxisWalk& walk, double* out, int* counted)
{
    const R* r = static_cast<const R*>(rho);
    const R* u[3] = { static_cast<const R*>(vx), static_cast<const R*>(vy), static_cast<const R*>(vz) };
    for (unsigned long long k = 0; k < N; ++k) {
        R v = R(0);
        counted[k] = enstrophyAtNode<R>(r, u[0], u[1], u[2], geo, walk, (uint32_t)k, v) ? 1 : 0;
        out[k] = counted[k] ? (double)v : 0.0;
    }
}
} // namespace
} // namespace vfb

using namespace vfb;

extern "C" int vfb_enstrophy(int precision, const void* rho, const void* vx, const void* vy, const void* vz,
                             unsigned long long N, const uint32_t* geo, const uint32_t* nX, const uint32_t* nY,
                             const uint32_t* nZ, const uint32_t* neighborInverse, double* out2, void* stream)
{
    clearError();
    if (!out2)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out2 is NULL");
    out2[0] = out2[1] = 0.0;
    if (!rho || !vx || !vy || !vz || !geo || !nX || !nY || !nZ || !neighborInverse)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (N < 2 || N > 0xffffffffull)
        return setError(VFB_ERR_OUT_OF_RANGE, "numberOfLBnodes %llu outside [2, 2^32)", N);
    if (precision != VFB_FP64 && precision != VFB_FP32)
        return setError(VFB_ERR_INVALID_ARGUMENT, "precision must be VFB_FP64 or VFB_FP32");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned blocks = (unsigned)sms * 4u;
    const unsigned long long need = (N + kEnstrophyThreads - 1) / kEnstrophyThreads;
    if (need < blocks)
        blocks = (unsigned)need;
    double* partial = nullptr;
    if (cudaMallocAsync(&partial, sizeof(double) * 2 * blocks, s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "cudaMallocAsync of %u partial sums failed", blocks);
    const AxisWalk walk { nX, nY, nZ, neighborInverse };
    if (precision == VFB_FP64)
        enstrophyKernel<double><<<blocks, kEnstrophyThreads, 0, s>>>(
            static_cast<const double*>(rho), static_cast<const double*>(vx), static_cast<const double*>(vy),
            static_cast<const double*>(vz), N, geo, walk, partial);
    else
        enstrophyKernel<float><<<blocks, kEnstrophyThreads, 0, s>>>(
            static_cast<const float*>(rho), static_cast<const float*>(vx), static_cast<const float*>(vy),
            static_cast<const float*>(vz), N, geo, walk, partial);
    int rc = checkLaunch("enstrophy");
    if (rc == VFB_OK) {
        std::vector<double> host(2 * (size_t)blocks);
        if (cudaMemcpyAsync(host.data(), partial, sizeof(double) * 2 * blocks, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = setError(VFB_ERR_CUDA, "copy of partial sums failed: %s", cudaGetErrorString(cudaGetLastError()));
        } else {
            double sum = 0.0, count = 0.0;
            for (unsigned b = 0; b < blocks; ++b) {
                sum += host[2 * b + 0];
                count += host[2 * b + 1];
            }
            out2[0] = count > 0.0 ? sum / count : 0.0;
            out2[1] = count;
        }
    }
    cudaFreeAsync(partial, s);
    return rc;
}

/*
 * The enstrophy node values on the host with the code the kernel runs (host
 * arrays): out[k] the value, counted[k] 1 where the node enters the mean.
 * For tests without a GPU.
 */
extern "C" int vfb_debug_enstrophy_nodes(int precision, const void* rho, const void* vx, const void* vy,
                                         const void* vz, unsigned long long N, const uint32_t* geo,
                                         const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
                                         const uint32_t* neighborInverse, double* out, int* counted)
{
    clearError();
    if (!rho || !vx || !vy || !vz || !geo || !nX || !nY || !nZ || !neighborInverse || !out || !counted)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    const AxisWalk walk { nX, nY, nZ, neighborInverse };
    if (precision == VFB_FP64)
        nodesOnHost<double>(rho, vx, vy, vz, N, geo, walk, out, counted);
    else if (precision == VFB_FP32)
        nodesOnHost<float>(rho, vx, vy, vz, N, geo, walk, out, counted);
    else
        return setError(VFB_ERR_INVALID_ARGUMENT, "precision must be VFB_FP64 or VFB_FP32");
    return VFB_OK;
}
