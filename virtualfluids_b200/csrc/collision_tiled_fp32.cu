// collision_tiled_fp32.cu -- the planned collision's kernels and launchers for
// FP32 storage (one translation unit per format, compiled in parallel).
#include "collision_tiled.cuh"

namespace vfb
{
int launchTiledFP32(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s)
{
    return launchTiled<float>(op, p, c, s);
}
} // namespace vfb
