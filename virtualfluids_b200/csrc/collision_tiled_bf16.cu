// collision_tiled_bf16.cu -- the planned collision's kernels and launchers for
// BF16 storage (one translation unit per format, compiled in parallel).
#include "collision_tiled.cuh"

namespace vfb
{
int launchTiledBF16(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s)
{
    return launchTiled<__nv_bfloat16>(op, p, c, s);
}
} // namespace vfb
