// Segment kernels: T_new on node layer runs (zalesak_limit b3, flux2dtracer_fct, ale_reconstruct). The bodies are in fct_segments.cuh; one translation
// unit per stage keeps the template instantiations of each stage compiling in parallel.
#include "fct_segments.cuh"

namespace fct {
namespace {

FCT_SEG_KERNEL(k_seg_final, seg_node_final)

#define FCT_COUNT(V) d.max_nseg[V]
FCT_SEG_LAUNCHER(launch_impl, k_seg_final, FCT_COUNT, FCT_GRID_N, FCT_GRID_1, kStageFinal)
#undef FCT_COUNT

}  // namespace

int launch_seg_final(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0, int c1,
                     cudaStream_t s) {
  return launch_impl(single, tab, n, d, c0, c1, s);
}

}  // namespace fct
