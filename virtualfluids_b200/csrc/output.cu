// output.cu -- the output pass of a level in one read of the populations.
//
// The reference's output path computes the macroscopic fields
// (calculateMacroscopicQuantitiesCompressible, PostProcessor/MacroscopicQuantities.cu,
// called from Simulation::readAndWriteFiles, Simulation.cpp:595-739) and, in
// separate passes, the kinetic-energy analyzer's mean (KineticEnergyAnalyzer::run,
// KineticEnergyAnalyzer.cu:66-154) and the enstrophy.  Here one kernel reads
// each node's 27 populations once and writes drho and u (the arithmetic of
// vfb_macroscopic) while it accumulates, in FP64, the sums of vfb_mass_and_energy
// over the fluid list and the analyzer's sum over its node set; a node's
// membership comes from a byte mask (bit 0 fluid list, bit 1 analyzer set).
// The enstrophy needs the velocity of neighbours and runs as a second kernel
// on the fields this one wrote.
#include <cuda_runtime.h>

#include <vector>

#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"

namespace vfb
{
namespace
{
constexpr int kOutThreads = 256;
constexpr int kSums = 5; // mass, energy, non-finite, analyzer energy, analyzer count

template <class S, bool EVEN>
__global__ void __launch_bounds__(kOutThreads)
    outputKernel(const S* __restrict__ dist, unsigned long long N, const uint32_t* __restrict__ geo,
                 const uint32_t* __restrict__ nX, const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                 const uint8_t* __restrict__ mask, typename Storage<S>::R* rho, typename Storage<S>::R* vx,
                 typename Storage<S>::R* vy, typename Storage<S>::R* vz, double* __restrict__ partial)
{
    using R = typename Storage<S>::R;
    double acc[kSums] = { 0.0, 0.0, 0.0, 0.0, 0.0 };
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < N;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t g = geo[k];
        if (g == 15u || g == 16u) {
            rho[k] = R(0);
            vx[k] = R(0);
            vy[k] = R(0);
            vz[k] = R(0);
            continue;
        }
        const Locs L = listIndices((uint32_t)k, nX, nY, nZ);
        R f[27];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], d);
        const R drho = pyramidDensity(f);
        const R oneOverRho = R(1) / (drho + R(1));
        const R ux = pyramidJx(f) * oneOverRho, uy = pyramidJy(f) * oneOverRho, uz = pyramidJz(f) * oneOverRho;
        rho[k] = drho;
        vx[k] = ux;
        vy[k] = uy;
        vz[k] = uz;
        const uint8_t m = mask[k];
        if (m) {
            const double dux = (double)ux, duy = (double)uy, duz = (double)uz;
            const double ke = 0.5 * (dux * dux + duy * duy + duz * duz) * ((double)drho + 1.0);
            const bool finite = isfinite(ke) && isfinite((double)drho);
            if (m & 1u) {
                if (finite) {
                    acc[0] += (double)drho;
                    acc[1] += ke;
                } else {
                    acc[2] += 1.0;
                }
            }
            if ((m & 2u) && finite) {
                acc[3] += ke;
                acc[4] += 1.0;
            }
        }
    }
    __shared__ double sm[kSums][kOutThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < kSums; ++i) {
        double v = acc[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0)
            sm[i][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < kSums) {
        double s = 0.0;
        for (int w = 0; w < kOutThreads / 32; ++w)
            s += sm[threadIdx.x][w];
        partial[(unsigned long long)kSums * blockIdx.x + threadIdx.x] = s;
    }
}

template <class S>
int launchOutput(const void* dist, unsigned long long N, const uint32_t* geo, const uint32_t* nX,
                 const uint32_t* nY, const uint32_t* nZ, const uint8_t* mask, int even, void* rho, void* vx,
                 void* vy, void* vz, double* partial, unsigned blocks, cudaStream_t s)
{
    using R = typename Storage<S>::R;
    const S* d = static_cast<const S*>(dist);
    R *r = static_cast<R*>(rho), *x = static_cast<R*>(vx), *y = static_cast<R*>(vy), *z = static_cast<R*>(vz);
    if (even)
        outputKernel<S, true><<<blocks, kOutThreads, 0, s>>>(d, N, geo, nX, nY, nZ, mask, r, x, y, z, partial);
    else
        outputKernel<S, false><<<blocks, kOutThreads, 0, s>>>(d, N, geo, nX, nY, nZ, mask, r, x, y, z, partial);
    return checkLaunch("output pass");
}
} // namespace
} // namespace vfb

using namespace vfb;

extern "C" int vfb_output_pass(int storage, const void* distributions, unsigned long long N, const uint32_t* geo,
                               const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ, const uint8_t* nodeMask,
                               int isEven, void* rho, void* vx, void* vy, void* vz, double* out5, void* stream)
{
    clearError();
    if (!out5)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out5 is NULL");
    for (int i = 0; i < kSums; ++i)
        out5[i] = 0.0;
    if (N == 0)
        return VFB_OK;
    if (!distributions || !geo || !nX || !nY || !nZ || !nodeMask || !rho || !vx || !vy || !vz)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned blocks = (unsigned)sms * 8u;
    const unsigned long long need = (N + kOutThreads - 1) / kOutThreads;
    if (need < blocks)
        blocks = (unsigned)need;
    double* partial = nullptr;
    if (cudaMallocAsync(&partial, sizeof(double) * kSums * blocks, s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "cudaMallocAsync of %u partial sums failed", blocks);
    int rc = VFB_OK;
    switch (storage) {
    case VFB_FP32: rc = launchOutput<float>(distributions, N, geo, nX, nY, nZ, nodeMask, isEven, rho, vx, vy, vz, partial, blocks, s); break;
    case VFB_FP64: rc = launchOutput<double>(distributions, N, geo, nX, nY, nZ, nodeMask, isEven, rho, vx, vy, vz, partial, blocks, s); break;
    case VFB_FP16: rc = launchOutput<__half>(distributions, N, geo, nX, nY, nZ, nodeMask, isEven, rho, vx, vy, vz, partial, blocks, s); break;
    case VFB_FX16: rc = launchOutput<int16_t>(distributions, N, geo, nX, nY, nZ, nodeMask, isEven, rho, vx, vy, vz, partial, blocks, s); break;
    case VFB_FX16W: rc = launchOutput<fx16w_t>(distributions, N, geo, nX, nY, nZ, nodeMask, isEven, rho, vx, vy, vz, partial, blocks, s); break;
    default: rc = launchOutput<__nv_bfloat16>(distributions, N, geo, nX, nY, nZ, nodeMask, isEven, rho, vx, vy, vz, partial, blocks, s); break;
    }
    if (rc == VFB_OK) {
        std::vector<double> host((size_t)kSums * blocks);
        if (cudaMemcpyAsync(host.data(), partial, sizeof(double) * kSums * blocks, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = setError(VFB_ERR_CUDA, "copy of partial sums failed: %s", cudaGetErrorString(cudaGetLastError()));
        } else {
            for (unsigned b = 0; b < blocks; ++b)
                for (int i = 0; i < kSums; ++i)
                    out5[i] += host[(size_t)kSums * b + i];
        }
    }
    cudaFreeAsync(partial, s);
    return rc;
}
