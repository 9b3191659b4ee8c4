// Segment kernels: limiter factors on node layer runs (zalesak_limit a1-a4, b1, b2). The bodies are in fct_segments.cuh; one translation
// unit per stage keeps the template instantiations of each stage compiling in parallel.
#include "fct_segments.cuh"

namespace fct {
namespace {

FCT_SEG_LIMIT_KERNEL(k_seg_limit)

#define FCT_COUNT(V) d.max_nseg[V]
FCT_SEG_LAUNCHER(launch_impl, k_seg_limit, FCT_COUNT, FCT_LIMIT_GRID_N, FCT_LIMIT_GRID_1, kStageLimit)
#undef FCT_COUNT

}  // namespace

int launch_seg_limit(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0, int c1,
                     cudaStream_t s) {
  return launch_impl(single, tab, n, d, c0, c1, s);
}

}  // namespace fct
