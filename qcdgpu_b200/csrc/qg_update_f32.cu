// FP32-link instantiations of the phase kernel (split from FP64 so the two
// compile in parallel).
#include "qg_update.cuh"
namespace qg {
cudaError_t launch_phase_f32(const Geom &G, void *links, int group, const PhaseArgs &a, cudaStream_t s)
{
    return launch_phase_T<float>(G, links, group, a, s);
}
}  // namespace qg
