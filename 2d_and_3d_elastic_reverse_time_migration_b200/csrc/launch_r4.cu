// Instantiation of the step kernels for stencil half-width R=4 (8th order).
#include "step_kernels_pair.cuh"

namespace ertm {

cudaError_t launch_stress_r4(const Geom& g, const KArgs& a, const StressMaps& m, bool cpml,
                             bool psplit, cudaStream_t s)
{
    return launch_stress_any<4>(g, a, m, cpml, psplit, s);
}

cudaError_t launch_velocity_r4(const Geom& g, const KArgs& a, const VelMaps& m, bool cpml, int epi,
                               bool record, cudaStream_t s)
{
    return launch_velocity_any<4>(g, a, m, cpml, epi, record, s);
}

cudaError_t launch_stress_multi_r4(dim3 grid, const StressMulti& P, bool cpml, cudaStream_t s)
{
    return launch_stress_multi_t<4>(grid, P, cpml, s);
}

cudaError_t launch_velocity_multi_r4(dim3 grid, const VelMulti& P, bool cpml, int epi, cudaStream_t s)
{
    return launch_velocity_multi_t<4>(grid, P, cpml, epi, s);
}

}  // namespace ertm
