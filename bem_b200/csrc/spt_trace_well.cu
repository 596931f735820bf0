// Trace and stage-evaluation kernels of geometry kind SPT_GEOM_WELL_BEM, every arithmetic
// form and far rule it offers (one translation unit per kind, so the kinds
// compile in parallel).
#include "spt_device.cuh"

namespace spt {
SPT_INSTANTIATE_KIND(SPT_GEOM_WELL_BEM)
}  // namespace spt
