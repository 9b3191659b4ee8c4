// Segment kernels: LO and adf_v on node layer runs (compute_fct_lo, adv_flux_ver_ho). The bodies are in fct_segments.cuh; one translation
// unit per stage keeps the template instantiations of each stage compiling in parallel.
#include "fct_segments.cuh"

namespace fct {
namespace {

FCT_SEG_KERNEL(k_seg_lo, seg_node_lo)

#define FCT_COUNT(V) d.max_nseg[V]
FCT_SEG_LAUNCHER(launch_impl, k_seg_lo, FCT_COUNT, FCT_GRID_N, FCT_GRID_1, kStageLo)
#undef FCT_COUNT

}  // namespace

int launch_seg_lo(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0, int c1,
                  cudaStream_t s) {
  return launch_impl(single, tab, n, d, c0, c1, s);
}

}  // namespace fct
