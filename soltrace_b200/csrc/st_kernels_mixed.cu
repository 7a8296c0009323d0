// Mixed FP32/FP64 instantiation of the trace kernels (fused multiply-add allowed).
#include "st_launch.h"
#include "st_trace_impl.cuh"

namespace stb {
void launch_probe_mixed(const SceneDev &S, uint64_t s0, uint32_t n, uint32_t *hit_elem, uint32_t *block_counts,
                       const RunState *rs, cudaStream_t st) {
    const uint32_t nb = (n + kProbeBlock - 1) / kProbeBlock;
    k_probe<1><<<nb, kProbeBlock, 0, st>>>(S, s0, n, hit_elem, block_counts, rs);
}
void launch_trace_mixed(bool records, const SceneDev &S, const uint64_t *hit_sid, const uint32_t *hit_el,
                       const uint32_t *hit_idx, const uint32_t *total, RunState *rs, const TraceOut &O,
                       uint32_t blocks, cudaStream_t st) {
    if (records)
        k_trace<1, 1><<<blocks, kTraceBlock, 0, st>>>(S, hit_sid, hit_el, hit_idx, total, rs, O);
    else
        k_trace<1, 0><<<blocks, kTraceBlock, 0, st>>>(S, hit_sid, hit_el, hit_idx, total, rs, O);
}
// resident trace blocks per SM, from this instantiation's register and shared-memory use
int trace_blocks_per_sm_mixed(bool records) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, records ? k_trace<1, 1> : k_trace<1, 0>, kTraceBlock, 0);
    return nb > 0 ? nb : 1;
}
}  // namespace stb
