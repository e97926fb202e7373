// mass_energy_static.cu -- the FP64 mass / kinetic-energy sums of
// vfb_mass_and_energy without any allocation.
//
// vfb_mass_and_energy takes its block partial sums from cudaMallocAsync.
// Some callers cannot allocate device memory at the point where they want the
// sums: a host that has handed the whole HBM to its own pool allocator and
// forbids allocations behind the pool's back, or a monitoring hook called
// from inside a solver loop whose memory footprint must stay fixed (a
// cudaMalloc there can fail late in a long run, or synchronise the device).
// vfb_mass_and_energy_static serves them: its scratch is a fixed array in the
// library's own device image, so the call allocates nothing, on the device or
// the host.
//
// The scratch holds partial sums for at most kStaticPartials blocks (24 KiB of
// doubles plus a result triple and a block counter).  Every GPU that loads the
// library keeps that array until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "capi_common.cuh"
#include "collision_math.cuh"
#include "d3q27.cuh"
#include "storage.cuh"

namespace vfb
{

constexpr unsigned kStaticPartials = 1024; // blocks whose partial sums the scratch holds
constexpr int kStaticThreads = 256;
constexpr int kMaxDevices = 64;

// partial[3 * b + i] for block b; result[0..2] the final sums; counter = number
// of blocks that have stored their partials in the current call.
struct StaticMassEnergyScratch {
    double partial[3 * kStaticPartials];
    double result[3];
    unsigned int counter;
};

// Host code sees only a stand-in for this symbol; its device address comes
// from cudaGetSymbolAddress (per device, see scratchOnCurrentDevice).
static __device__ __align__(256) StaticMassEnergyScratch gMassEnergyScratch;

template <class S, bool EVEN>
__global__ void __launch_bounds__(kStaticThreads)
    massEnergyStaticKernel(const S* __restrict__ dist, unsigned long long N, const uint32_t* __restrict__ nX,
                           const uint32_t* __restrict__ nY, const uint32_t* __restrict__ nZ,
                           const uint32_t* __restrict__ idx, uint32_t n, StaticMassEnergyScratch* scratch)
{
    using R = typename Storage<S>::R;
    double m = 0.0, e = 0.0, bad = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = __ldg(idx + i);
        const Locs L = listIndices(k, nX, nY, nZ);
        R f[27];
#pragma unroll
        for (int d = 0; d < 27; ++d)
            f[d] = Storage<S>::load(dist + (unsigned long long)slot<EVEN>(d) * N + L.k[loc(d)], d);
        const R drho = pyramidDensity(f);
        const R oneOverRho = R(1) / (drho + R(1));
        const double ux = (double)(pyramidJx(f) * oneOverRho);
        const double uy = (double)(pyramidJy(f) * oneOverRho);
        const double uz = (double)(pyramidJz(f) * oneOverRho);
        const double ke = 0.5 * (ux * ux + uy * uy + uz * uz) * ((double)drho + 1.0);
        if (isfinite(ke) && isfinite((double)drho)) {
            m += (double)drho;
            e += ke;
        } else {
            bad += 1.0;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        e += __shfl_down_sync(0xffffffffu, e, o);
        bad += __shfl_down_sync(0xffffffffu, bad, o);
    }
    __shared__ double sm[3][kStaticThreads / 32];
    __shared__ bool lastBlock;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sm[0][warp] = m;
        sm[1][warp] = e;
        sm[2][warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
        m = lane < kStaticThreads / 32 ? sm[0][lane] : 0.0;
        e = lane < kStaticThreads / 32 ? sm[1][lane] : 0.0;
        bad = lane < kStaticThreads / 32 ? sm[2][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m += __shfl_down_sync(0xffffffffu, m, o);
            e += __shfl_down_sync(0xffffffffu, e, o);
            bad += __shfl_down_sync(0xffffffffu, bad, o);
        }
        if (lane == 0) {
            scratch->partial[3 * blockIdx.x + 0] = m;
            scratch->partial[3 * blockIdx.x + 1] = e;
            scratch->partial[3 * blockIdx.x + 2] = bad;
            __threadfence();
            // the block that stores the last partial sums them all (no block waits for another)
            lastBlock = atomicAdd(&scratch->counter, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (lastBlock && threadIdx.x == 0) {
        __threadfence();
        const volatile double* p = scratch->partial;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        // block order, as vfb_mass_and_energy sums its partials on the host
        for (unsigned b = 0; b < gridDim.x; ++b) {
            s0 += p[3 * b + 0];
            s1 += p[3 * b + 1];
            s2 += p[3 * b + 2];
        }
        scratch->result[0] = s0;
        scratch->result[1] = s1;
        scratch->result[2] = s2;
        scratch->counter = 0u; // ready for the next call on this device
    }
}

// Device address of the scratch on the current device, looked up once per
// device; nullptr (and the error recorded) if the lookup fails.  The address
// is that of the device's context at the first call: a cudaDeviceReset
// destroys that context, after which the cached address is stale (the header
// tells callers not to use the entry point on a device after a reset).
static StaticMassEnergyScratch* scratchOnCurrentDevice()
{
    static std::mutex lock;
    static StaticMassEnergyScratch* address[kMaxDevices] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
        setError(VFB_ERR_CUDA, "no usable current device (%d)", device);
        return nullptr;
    }
    std::lock_guard<std::mutex> guard(lock);
    if (!address[device]) {
        StaticMassEnergyScratch* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), gMassEnergyScratch);
        if (rc != cudaSuccess || !p) {
            setError(VFB_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed on device %d: %s", device,
                     cudaGetErrorString(rc));
            return nullptr;
        }
        address[device] = p;
    }
    return address[device];
}

template <class S>
static int launchStatic(const void* dist, unsigned long long N, const uint32_t* nX, const uint32_t* nY,
                        const uint32_t* nZ, const uint32_t* idx, uint32_t n, int even, unsigned blocks,
                        StaticMassEnergyScratch* scratch, cudaStream_t stream)
{
    if (even)
        massEnergyStaticKernel<S, true><<<blocks, kStaticThreads, 0, stream>>>(static_cast<const S*>(dist), N, nX,
                                                                              nY, nZ, idx, n, scratch);
    else
        massEnergyStaticKernel<S, false><<<blocks, kStaticThreads, 0, stream>>>(static_cast<const S*>(dist), N, nX,
                                                                               nY, nZ, idx, n, scratch);
    return checkLaunch("mass and energy (static scratch)");
}

} // namespace vfb

using namespace vfb;

extern "C" int vfb_mass_and_energy_static(int storage, const void* distributions, unsigned long long N,
                                          const uint32_t* nX, const uint32_t* nY, const uint32_t* nZ,
                                          const uint32_t* idx, uint32_t n, int isEven, double* out, void* stream)
{
    clearError();
    if (!out)
        return setError(VFB_ERR_INVALID_ARGUMENT, "out is NULL");
    out[0] = out[1] = out[2] = 0.0;
    if (n == 0)
        return VFB_OK;
    if (!distributions || !nX || !nY || !nZ || !idx)
        return setError(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    if (vfb_storage_bytes(storage) == 0)
        return setError(VFB_ERR_INVALID_ARGUMENT, "unknown storage %d", storage);
    StaticMassEnergyScratch* scratch = scratchOnCurrentDevice();
    if (!scratch)
        return VFB_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned blocks = (unsigned)sms * 4u;
    const unsigned need = (n + kStaticThreads - 1) / kStaticThreads;
    if (need < blocks)
        blocks = need;
    if (blocks > kStaticPartials)
        return setError(VFB_ERR_OUT_OF_RANGE,
                        "the launch needs %u block partial sums but the static scratch holds %u "
                        "(4 blocks per SM on GPUs with up to %u SMs)",
                        blocks, kStaticPartials, kStaticPartials / 4);
    // the block counter must start at zero; the last block of every call resets
    // it, and clearing it here also recovers from a call that never finished
    if (cudaMemsetAsync(&scratch->counter, 0, sizeof(unsigned int), s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "clearing the block counter failed: %s",
                        cudaGetErrorString(cudaGetLastError()));
    int rc = VFB_OK;
    switch (storage) {
    case VFB_FP32: rc = launchStatic<float>(distributions, N, nX, nY, nZ, idx, n, isEven, blocks, scratch, s); break;
    case VFB_FP64: rc = launchStatic<double>(distributions, N, nX, nY, nZ, idx, n, isEven, blocks, scratch, s); break;
    case VFB_FP16: rc = launchStatic<__half>(distributions, N, nX, nY, nZ, idx, n, isEven, blocks, scratch, s); break;
    case VFB_FX16: rc = launchStatic<int16_t>(distributions, N, nX, nY, nZ, idx, n, isEven, blocks, scratch, s); break;
    case VFB_FX16W: rc = launchStatic<fx16w_t>(distributions, N, nX, nY, nZ, idx, n, isEven, blocks, scratch, s); break;
    default: rc = launchStatic<__nv_bfloat16>(distributions, N, nX, nY, nZ, idx, n, isEven, blocks, scratch, s); break;
    }
    if (rc != VFB_OK)
        return rc;
    double result[3];
    if (cudaMemcpyAsync(result, scratch->result, sizeof(result), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return setError(VFB_ERR_CUDA, "copy of the sums failed: %s", cudaGetErrorString(cudaGetLastError()));
    out[0] = result[0];
    out[1] = result[1];
    out[2] = result[2];
    return VFB_OK;
}
