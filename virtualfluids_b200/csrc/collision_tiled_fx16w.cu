// collision_tiled_fx16w.cu -- the planned collision's kernels and launchers for
// FX16W storage (one translation unit per format, compiled in parallel).
#include "collision_tiled.cuh"

namespace vfb
{
int launchTiledFX16W(Op op, const vfb_collision_plan_impl& p, const vfb_collision_args* c, cudaStream_t s)
{
    return launchTiled<fx16w_t>(op, p, c, s);
}
} // namespace vfb
