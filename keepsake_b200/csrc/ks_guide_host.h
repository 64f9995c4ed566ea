// Host-side entry points of the guide network used by the integrator (ks_guide is opaque there).
#pragma once
#include "../../include/ks_b200.h"
#include <cuda_runtime.h>

namespace ksb
{
namespace guide_impl
{
ks_context *context_of(const ks_guide *g);
// Mixtures for the paths of a wavefront hit queue (count read on the device, at most max_rows,
// which sizes the grid), written per path slot into lobes (10 float4 per slot, cap slots apart), on
// `stream` (null: the guide's context stream).
ks_status infer_paths(ks_guide *g, const uint32_t *queue, const uint32_t *queue_count, const float4 *o_pdf,
                      const float4 *d_info, const float4 *hits, const float4 *prim_tris, const uint32_t *hit_inst,
                      const float *inst_xf, float4 *lobes, uint32_t cap, uint32_t max_rows,
                      cudaStream_t stream = nullptr);
// Adam steps over n device-resident training rows in batches of `batch`; *steps counts them.  The
// w component of each wo row holds the BSDF pdf of the row's wi.
ks_status train_rows(ks_guide *g, uint32_t n, const float4 *pos, const float4 *wo, const float4 *nrm,
                     const float4 *wi, const float *t, uint32_t batch, uint32_t *steps);
// KS_OK unless a tensor-core wait of an earlier launch timed out (synchronises the stream).
ks_status status(ks_guide *g);
} // namespace guide_impl
} // namespace ksb
