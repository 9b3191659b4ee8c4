// Segment kernels: adf_h on edge level runs (fill_up_dn_grad, adv_flux_hor_ho), plus the lane kernel of the remaining edge lanes. The bodies are in fct_segments.cuh; one translation
// unit per stage keeps the template instantiations of each stage compiling in parallel.
#include "fct_segments.cuh"

namespace fct {
namespace {

FCT_SEG_KERNEL(k_seg_edge, seg_edge_adf)

// the remaining edge lanes: one lane per thread (tracer slices as in the segment kernels)
template <int NTR>
__global__ void __launch_bounds__(256) k_edge_fix_1(Inst in, int t0, int w0) {
  const int sub = int(blockIdx.y) * NTR;
  body_edge_fix<NTR, false>(in, lane_index(), t0 + sub, w0 + sub);
}
template <int NTR>
__global__ void __launch_bounds__(256) k_edge_fix_n(const Inst* __restrict__ tab, int t0, int w0,
                                                    int lg) {
  const int64_t g = lane_index();
  const int sub = int(g & ((int64_t(1) << lg) - 1)) * NTR;
  body_edge_fix<NTR, true>(tab[blockIdx.y], g >> lg, t0 + sub, w0 + sub);
}

}  // namespace

int launch_edge_fix(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0,
                    int c1, cudaStream_t s) {
  if (d.max_efix == 0) return FCT_OK;
  for (int t0 = c0; t0 < c1;) {
    const int rem = c1 - t0;
    const int P = seg_tracers(rem, d.smap_tracers[kStageEdge], tab != nullptr, 1, seg_even(d));
    int lg = 0;
    while (lg < 3 && (P << (lg + 1)) <= rem) ++lg;
    const int w0 = t0 - c0;
    if (tab) {
      const dim3 g(seg_blocks(d.max_efix << lg), unsigned(n));
      if (P == 4) k_edge_fix_n<4><<<g, 256, 0, s>>>(tab, t0, w0, lg);
      else if (P == 2) k_edge_fix_n<2><<<g, 256, 0, s>>>(tab, t0, w0, lg);
      else k_edge_fix_n<1><<<g, 256, 0, s>>>(tab, t0, w0, lg);
    } else {
      const dim3 g(seg_blocks(d.max_efix), 1u << lg);
      if (P == 2) k_edge_fix_1<2><<<g, 256, 0, s>>>(single, t0, w0);
      else k_edge_fix_1<1><<<g, 256, 0, s>>>(single, t0, w0);
    }
    t0 += P << lg;
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? FCT_OK : cuda_error(e, "launch_edge_fix");
}

namespace {

#define FCT_COUNT(V) d.max_eseg[V]
FCT_SEG_LAUNCHER(launch_impl, k_seg_edge, FCT_COUNT, FCT_GRID_N, FCT_GRID_1, kStageEdge)
#undef FCT_COUNT

}  // namespace

int launch_seg_edge(const Inst& single, const Inst* tab, int n, const LaunchDims& d, int c0, int c1,
                    cudaStream_t s) {
  return launch_impl(single, tab, n, d, c0, c1, s);
}

}  // namespace fct
