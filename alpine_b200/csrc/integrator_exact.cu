// Integrator kernels compiled without multiply-add contraction (-fmad=false,
// set by the build for *_exact.cu), so every FP32 product and sum is rounded
// separately, as in the reference compiled with -ffp-contract=off. Used with
// the reference RNG stream for image parity (see integrator.cuh).
#define AG_INTEGRATOR_NS exact
#include "integrator.cuh"

namespace ag {
const IntegratorKernels& integrator_exact()
{
    static const IntegratorKernels k = {exact::generate, exact::shade, exact::resolve, exact::accumulate,
                                              exact::guide_query, exact::train_finalize,
                                              exact::sort};
    return k;
}
}  // namespace ag
