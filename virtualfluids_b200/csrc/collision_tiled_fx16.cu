// collision_tiled_fx16.cu -- the planned collision's kernels and launchers for
// FX16 storage (one translation unit per format, compiled in parallel).
#include "collision_tiled.cuh"

namespace vfb
{
int launchTiledFX16(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s)
{
    return launchTiled<int16_t>(op, p, c, s);
}
} // namespace vfb
