// Integrator kernels, default floating-point flags (see integrator.cuh).
#define AG_INTEGRATOR_NS fast
#include "integrator.cuh"

namespace ag {
const IntegratorKernels& integrator_fast()
{
    static const IntegratorKernels k = {fast::generate, fast::shade, fast::resolve, fast::accumulate,
                                              fast::guide_query, fast::train_finalize,
                                              fast::sort};
    return k;
}
}  // namespace ag
