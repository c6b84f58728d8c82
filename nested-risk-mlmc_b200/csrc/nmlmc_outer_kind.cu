// Instantiations of the batched level sequence for one sampler kind (NMLMC_OUTER_KIND = 0
// reference model, 1 shift model, 2 portfolio, 4 portfolio with path-simulated options), in all
// three precisions; compiled once per kind.
#include "nmlmc_outer_impl.cuh"

#ifndef NMLMC_OUTER_KIND
#error "NMLMC_OUTER_KIND must be defined (0, 1, 2 or 4)"
#endif

namespace nmlmc {

template cudaError_t sample_level_t<float, NMLMC_OUTER_KIND, PREC_FP32>(const OuterLevel<float>&, OuterBuffers&,
                                                                        TraceRec*, cudaStream_t);
template cudaError_t sample_level_t<float, NMLMC_OUTER_KIND, PREC_REF32>(const OuterLevel<float>&, OuterBuffers&,
                                                                         TraceRec*, cudaStream_t);
template cudaError_t sample_level_t<double, NMLMC_OUTER_KIND, PREC_FP64>(const OuterLevel<double>&, OuterBuffers&,
                                                                         TraceRec*, cudaStream_t);

}  // namespace nmlmc
