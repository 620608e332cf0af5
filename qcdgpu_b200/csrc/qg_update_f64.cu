// FP64-link instantiations of the phase kernel.
#include "qg_update.cuh"
namespace qg {
cudaError_t launch_phase_f64(const Geom &G, void *links, int group, const PhaseArgs &a, cudaStream_t s)
{
    return launch_phase_T<double>(G, links, group, a, s);
}
}  // namespace qg
